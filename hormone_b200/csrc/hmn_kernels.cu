// hmn_kernels.cu -- FP64 kernels of the explicit MHD step for sm_100a.
//
// Compiled with --fmad=false: every operation is a single IEEE binary64
// operation in the reference's order, so results are bit-identical to the
// Fortran path (and to the CPU oracle that restates it).
//
// State in HBM (per simulation, interior cells only, x fastest):
//   U planes  (nvar):  rho, m1, m2, m3, E, B1, B2, B3, phi   (conserved)
//   P planes  (10):    rho, v1, v2, v3, e, B1, B2, B3, phi, eint
// P is what HORMONE keeps in module physval after `primitive`/`pressure`
// (rungekutta.f90:193-232, eos.f90:742-842); every stage writes the P of
// its output so the next stage reads primitives without dividing again.
//
// One RK stage (hydro.f90:35-41: boundarycondition -> numflux -> source ->
// rungekutta) is ONE launch of stage_kernel.  A CTA owns a tile of 256 cells:
//   1. it stages the primitives of the tile and of two cells beyond each face
//      of the tile (a cross-shaped region, no corners) into shared memory,
//      forming ghost cells from the boundary codes on the fly
//      (boundarycondition.f90, codes 0-3 and the ghost energy of :222-243);
//   2. per solved axis it computes the limited slopes (interpolation.f90),
//      the HLLD face fluxes (numflux.f90 + hlldflux.f90) and adds the flux
//      divergence of its cell to registers;
//   3. it applies the RK combination (rungekutta.f90:35-59) with the gravity
//      source (source.f90:70-85) and writes U and P of the new state.
// Slopes and fluxes never leave the SM.
#include <cuda_runtime.h>

#include <cstring>

#include <cstdint>
#include <cstdlib>

#include "hmn_face.cuh"
#include "hmn_internal.h"
#include "hmn_math.cuh"
#include "hmn_stage.cuh"
#include "hmn_queue.cuh"
#include "hmn_tile.cuh"

namespace hmn {

template <bool MAG, bool GLM, class TL, bool SPH = false, bool PUSH = false>
__global__ void __launch_bounds__(TL::NT, TL::MINB) stage_kernel(const GridDev G, const StageArgs A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SmemT<TL>& sm = *reinterpret_cast<SmemT<TL>*>(smem_raw);
  if (A.sc->done) return;
  stage_tile_exact<MAG, GLM, TL, SPH, PUSH>(G, A, sm, blockIdx.x, nullptr);
}

// the same stage with the stencil region staged by TMA (3-D tiles)
template <bool MAG, bool GLM, class TL>
__global__ void __launch_bounds__(TL::NT, TL::MINB)
    stage_kernel_tma(const GridDev G, const StageArgs A, const __grid_constant__ TmaMaps tm) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SmemT<TL>& sm = *reinterpret_cast<SmemT<TL>*>(smem_raw);
  if (A.sc->done) return;
  // bulk tensor copies need 128-byte aligned destinations (uniform over the CTA)
  const bool tma = (smem_addr(&sm.P[0][0]) & 127u) == 0;
  stage_tile_exact<MAG, GLM, TL>(G, A, sm, blockIdx.x, tma ? &tm : nullptr);
}

// ---------------------------------------------------------------------------
// P planes from the uploaded primitives (pressure at start-up, eos.f90:805-842)

template <bool MAG>
__global__ void prim_init_kernel(double* P, size_t plane) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < plane; c += (size_t)gridDim.x * blockDim.x) {
    const double d = P[c], v1 = P[plane + c], v2 = P[2 * plane + c], v3 = P[3 * plane + c];
    const double e = P[4 * plane + c];
    const double b1 = MAG ? P[5 * plane + c] : 0.0, b2 = MAG ? P[6 * plane + c] : 0.0;
    const double b3 = MAG ? P[7 * plane + c] : 0.0;
    P[PEINT * plane + c] = get_eint<MAG>(e, d, v1, v2, v3, b1, b2, b3);
  }
}

// P planes from conserved variables (rungekutta.f90:205-229 + eos.f90:805-842)
template <bool MAG, bool GLM>
__global__ void prim_from_u_kernel(const double* U, double* P, size_t plane) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < plane; c += (size_t)gridDim.x * blockDim.x) {
    const double d = U[c];
    const double v1 = U[plane + c] / d, v2 = U[2 * plane + c] / d, v3 = U[3 * plane + c] / d;
    const double e = U[4 * plane + c];
    const double b1 = MAG ? U[5 * plane + c] : 0.0, b2 = MAG ? U[6 * plane + c] : 0.0;
    const double b3 = MAG ? U[7 * plane + c] : 0.0;
    P[c] = d;
    P[plane + c] = v1;
    P[2 * plane + c] = v2;
    P[3 * plane + c] = v3;
    P[4 * plane + c] = e;
    P[5 * plane + c] = b1;
    P[6 * plane + c] = b2;
    P[7 * plane + c] = b3;
    P[8 * plane + c] = GLM ? U[8 * plane + c] : 0.0;
    P[PEINT * plane + c] = get_eint<MAG>(e, d, v1, v2, v3, b1, b2, b3);
  }
}

template <bool MAG>
__global__ void __launch_bounds__(256) cfl_kernel(const GridDev G, const double* P, size_t plane, double gamma,
                                                  DevScalars* sc) {
  if (sc->done) return;
  double my_dti = __longlong_as_double(0x7ff0000000000000LL);  // +inf
  double my_cf = 0.0;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < plane; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % G.n[0]);
    const int j = (int)((c / G.n[0]) % G.n[1]);
    const int k = (int)(c / ((size_t)G.n[0] * G.n[1]));
    double dti, cfm;
    if (!cfl_cell<MAG>(G, P, plane, gamma, c, i, j, k, sc, dti, cfm)) continue;
    my_cf = fmax2(my_cf, cfm);
    my_dti = fmin2(my_dti, dti);
  }
  cfl_block_reduce(my_dti, my_cf, sc);
}


__global__ void cfl_finalize_kernel(DevScalars* sc) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || sc->done) return;
  finalize_dt(sc);
}

// primitives of the current state for download: 9 planes (phi with the
// pending phidamp factor) and the gas pressure
__global__ void prim_out_kernel(const double* P, size_t plane, double phifac, double gm1, double* out,
                                double* p_out) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < plane; c += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < 8; q++) out[q * plane + c] = P[q * plane + c];
    out[8 * plane + c] = P[8 * plane + c] * phifac;
    if (p_out) p_out[c] = gm1 * P[PEINT * plane + c];
  }
}

// time += dt; tn += 1; end check (hormone.f90:147-155) on the device clock
__global__ void advance_kernel(DevScalars* sc) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || sc->done) return;
  sc->time = sc->time + sc->dt;
  sc->tn = sc->tn + 1;
  if (sc->endstyle == 1 && sc->time >= sc->t_end) sc->done = 1;
}

// ---------------------------------------------------------------------------
// host-side launchers (called from hmn_capi.cu)

// spherical grids: the plain (non-TMA) FP64 kernel with the metric factors
template <bool MAG, bool GLM, class TL>
static cudaError_t launch_stage_sph(const GridDev& G, const StageArgs& A, cudaStream_t st) {
  constexpr int smem = (int)sizeof(SmemT<TL>);
  const int blocks = A.tiles[0] * A.tiles[1] * A.tiles[2];
  static bool attr = false;
  if (!attr) {
    cudaError_t e =
        cudaFuncSetAttribute(stage_kernel<MAG, GLM, TL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  stage_kernel<MAG, GLM, TL, true><<<blocks, TL::NT, smem, st>>>(G, A);
  return cudaGetLastError();
}

// r always solved; 1-D grids carry no GLM wave, 2-D and 3-D MHD grids do
template <class TL>
static cudaError_t launch_stage_sph_tl(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st) {
  constexpr bool multi = (TL::TY > 1) || (TL::TZ > 1);
  if (mag && glm != multi) return cudaErrorInvalidValue;
  if (!mag) return launch_stage_sph<false, false, TL>(G, A, st);
  return launch_stage_sph<true, multi, TL>(G, A, st);
}

static cudaError_t launch_stage_spherical(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st) {
  const int* t = A.tile;
  if (A.nspc > 0) return cudaErrorInvalidValue;
  if (t[0] == 8 && t[1] == 8 && t[2] == 8) return launch_stage_sph_tl<Tile<8, 8, 8, 640, 1>>(G, A, mag, glm, st);
  if (t[0] == 8 && t[1] == 8 && t[2] == 4) return launch_stage_sph_tl<Tile<8, 8, 4, 384, 2>>(G, A, mag, glm, st);
  if (t[0] == 16 && t[1] == 16 && t[2] == 1) return launch_stage_sph_tl<Tile<16, 16, 1, 288, 2>>(G, A, mag, glm, st);
  if (t[0] == 16 && t[1] == 1 && t[2] == 16) return launch_stage_sph_tl<Tile<16, 1, 16, 288, 2>>(G, A, mag, glm, st);
  if (t[0] == 256 && t[1] == 1 && t[2] == 1) return launch_stage_sph_tl<Tile<256, 1, 1, 288, 2>>(G, A, mag, glm, st);
  return cudaErrorInvalidValue;
}

template <bool MAG, bool GLM, class TL>
static cudaError_t launch_stage_t(const GridDev& G, const StageArgs& A, const TmaMaps* tm, cudaStream_t st) {
  constexpr int smem = (int)sizeof(SmemT<TL>);
  const int blocks = A.tiles[0] * A.tiles[1] * A.tiles[2];
  if constexpr (TL::HX && TL::HY && TL::HZ) {  // TMA staging needs halos on all three axes
    if (tm != nullptr) {
      static bool attr_tma = false;
      if (!attr_tma) {
        cudaError_t e = cudaFuncSetAttribute(stage_kernel_tma<MAG, GLM, TL>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr_tma = true;
      }
      stage_kernel_tma<MAG, GLM, TL><<<blocks, TL::NT, smem, st>>>(G, A, *tm);
      return cudaGetLastError();
    }
  }
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<MAG, GLM, TL>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  stage_kernel<MAG, GLM, TL><<<blocks, TL::NT, smem, st>>>(G, A);
  return cudaGetLastError();
}

template <class TL>
static cudaError_t launch_stage_tl(const GridDev& G, const StageArgs& A, bool mag, bool glm, const TmaMaps* tm,
                                   cudaStream_t st) {
  if (mag && glm) return launch_stage_t<true, true, TL>(G, A, tm, st);
  if (mag) return launch_stage_t<true, false, TL>(G, A, tm, st);
  return launch_stage_t<false, false, TL>(G, A, tm, st);
}

// tile shapes by solved axes: 3-D 8x8x8 for FP64 (one CTA of 640 threads per
// SM) and 8x8x4 for the mixed form (two CTAs per SM), either one forced by
// HMN_TILE3D=888 or 884, and 8x8x4 whenever there are passive scalars;
// 2-D 16x16, 1-D 256
void stage_tile(const int solve[3], int precision, int nspc, int tile[3], bool sph) {
  const int dim = solve[0] + solve[1] + solve[2];
  for (int a = 0; a < 3; a++) tile[a] = 1;
  if (dim == 3 && nspc > 0) {  // the scalar planes only fit the smaller tile
    tile[0] = 8;
    tile[1] = 8;
    tile[2] = 4;
  } else if (dim == 3) {
    // 8x8x4 (two CTAs of 384 threads per SM) for the mixed form and for
    // spherical grids (the 160x80x160 polytrope: 467 against 442 M
    // zone-updates/s with 8x8x8); 8x8x8 for the FP64 tile otherwise, which
    // 3-D Cartesian grids only use with the march switched off
    const char* env = getenv("HMN_TILE3D");
    bool t884 = precision == 1 || sph;
    if (env && env[0] == '8' && env[1] == '8' && (env[2] == '4' || env[2] == '8')) t884 = env[2] == '4';
    tile[0] = 8;
    tile[1] = 8;
    tile[2] = t884 ? 4 : 8;
  } else {
    for (int a = 0; a < 3; a++)
      if (solve[a]) tile[a] = dim == 2 ? 16 : 256;
  }
}

// z slabs exchanging by push: the stage kernel also stores its two
// boundary layers into the neighbours' halo buffers (3-D Cartesian tiles)
template <bool MAG, bool GLM, class TL>
static cudaError_t launch_stage_push_t(const GridDev& G, const StageArgs& A, cudaStream_t st) {
  constexpr int smem = (int)sizeof(SmemT<TL>);
  const int blocks = A.tiles[0] * A.tiles[1] * A.tiles[2];
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<MAG, GLM, TL, false, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  stage_kernel<MAG, GLM, TL, false, true><<<blocks, TL::NT, smem, st>>>(G, A);
  return cudaGetLastError();
}

template <class TL>
static cudaError_t launch_stage_push_tl(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st) {
  if (mag && glm) return launch_stage_push_t<true, true, TL>(G, A, st);
  if (mag) return launch_stage_push_t<true, false, TL>(G, A, st);
  return launch_stage_push_t<false, false, TL>(G, A, st);
}

static cudaError_t launch_stage_push(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st) {
  const int* t = A.tile;
  if (G.sph.on || t[2] == 1) return cudaErrorInvalidValue;
  if (A.nspc > 4) return launch_stage_push_tl<Tile<8, 8, 4, 384, 1, 8>>(G, A, mag, glm, st);
  if (A.nspc > 0) return launch_stage_push_tl<Tile<8, 8, 4, 384, 2, 4>>(G, A, mag, glm, st);
  if (t[0] == 8 && t[1] == 8 && t[2] == 8) return launch_stage_push_tl<Tile<8, 8, 8, 640, 1>>(G, A, mag, glm, st);
  if (t[0] == 8 && t[1] == 8 && t[2] == 4) return launch_stage_push_tl<Tile<8, 8, 4, 384, 2>>(G, A, mag, glm, st);
  return cudaErrorInvalidValue;
}

// The stage tiles whose shared-memory layout has room for SP passive
// scalars (8 x 8 x 4 in 3-D; with 8 scalars its 203 KB allow one CTA per SM)
template <int SP, int MINB3>
static cudaError_t launch_scalar_tiles(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st) {
  const int* t = A.tile;
  if (t[0] == 8 && t[1] == 8 && t[2] == 4)
    return launch_stage_tl<Tile<8, 8, 4, 384, MINB3, SP>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 16 && t[1] == 16 && t[2] == 1)
    return launch_stage_tl<Tile<16, 16, 1, 288, MINB3, SP>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 16 && t[1] == 1 && t[2] == 16)
    return launch_stage_tl<Tile<16, 1, 16, 288, MINB3, SP>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 16 && t[2] == 16)
    return launch_stage_tl<Tile<1, 16, 16, 288, MINB3, SP>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 256 && t[1] == 1 && t[2] == 1) return launch_stage_tl<Tile<256, 1, 1, 288, 2, SP>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 256 && t[2] == 1) return launch_stage_tl<Tile<1, 256, 1, 288, 2, SP>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 1 && t[2] == 256) return launch_stage_tl<Tile<1, 1, 256, 288, 2, SP>>(G, A, mag, glm, nullptr, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage(const GridDev& G, const StageArgs& A, bool mag, bool glm, const TmaMaps* tm,
                         cudaStream_t st) {
  {
    const cudaError_t e = launch_stage_march(G, A, mag, glm, st);
    if (e != cudaErrorNotSupported) return e;
  }
  if (A.push[0] != nullptr || A.push[1] != nullptr) return launch_stage_push(G, A, mag, glm, st);
  if (G.sph.on) return launch_stage_spherical(G, A, mag, glm, st);
  const int* t = A.tile;
  if (A.nspc > 0) {  // tiles with room for up to 4, or up to 8, passive scalars
    if (A.nspc <= 4) return launch_scalar_tiles<4, 2>(G, A, mag, glm, st);
    return launch_scalar_tiles<8, 1>(G, A, mag, glm, st);
  }
  if (t[0] == 8 && t[1] == 8 && t[2] == 8) return launch_stage_tl<Tile<8, 8, 8, 640, 1>>(G, A, mag, glm, tm, st);
  if (t[0] == 8 && t[1] == 8 && t[2] == 4) return launch_stage_tl<Tile<8, 8, 4, 384, 2>>(G, A, mag, glm, tm, st);
  if (t[0] == 16 && t[1] == 16 && t[2] == 1) return launch_stage_tl<Tile<16, 16, 1, 288, 3>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 16 && t[1] == 1 && t[2] == 16) return launch_stage_tl<Tile<16, 1, 16, 288, 3>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 16 && t[2] == 16) return launch_stage_tl<Tile<1, 16, 16, 288, 3>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 256 && t[1] == 1 && t[2] == 1) return launch_stage_tl<Tile<256, 1, 1, 288, 3>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 256 && t[2] == 1) return launch_stage_tl<Tile<1, 256, 1, 288, 3>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 1 && t[2] == 256) return launch_stage_tl<Tile<1, 1, 256, 288, 3>>(G, A, mag, glm, nullptr, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_cfl_cells(const GridDev& G, const double* P, size_t plane, double gamma, DevScalars* sc,
                             bool mag, int nblocks, cudaStream_t st) {
  if (mag)
    cfl_kernel<true><<<nblocks, 256, 0, st>>>(G, P, plane, gamma, sc);
  else
    cfl_kernel<false><<<nblocks, 256, 0, st>>>(G, P, plane, gamma, sc);
  return cudaGetLastError();
}

cudaError_t launch_cfl_finalize(DevScalars* sc, cudaStream_t st) {
  cfl_finalize_kernel<<<1, 32, 0, st>>>(sc);
  return cudaGetLastError();
}

// send_lo[p][l][j][i] = P[p][k=l], send_hi[p][l][j][i] = P[p][k=nz-2+l]
__global__ void pack_zhalos_kernel(const double* P, int nx, int ny, int nz, int nplanes, double* send_lo,
                                   double* send_hi) {
  const size_t hp = (size_t)nx * ny, plane = hp * nz;
  const size_t total = (size_t)nplanes * 2 * hp;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const size_t p = t / (2 * hp), r = t % (2 * hp);
    const size_t l = r / hp, c = r % hp;
    if (send_lo) send_lo[t] = P[p * plane + l * hp + c];
    if (send_hi) send_hi[t] = P[p * plane + ((size_t)nz - 2 + l) * hp + c];
  }
}

cudaError_t launch_pack_zhalos(const double* P, const int n[3], int nplanes, double* send_lo, double* send_hi,
                               int nblocks, cudaStream_t st) {
  pack_zhalos_kernel<<<nblocks, 256, 0, st>>>(P, n[0], n[1], n[2], nplanes, send_lo, send_hi);
  return cudaGetLastError();
}

cudaError_t launch_cfl(const GridDev& G, const double* P, size_t plane, double gamma, DevScalars* sc, bool mag,
                       int nblocks, cudaStream_t st) {
  if (mag)
    cfl_kernel<true><<<nblocks, 256, 0, st>>>(G, P, plane, gamma, sc);
  else
    cfl_kernel<false><<<nblocks, 256, 0, st>>>(G, P, plane, gamma, sc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  cfl_finalize_kernel<<<1, 32, 0, st>>>(sc);
  return cudaGetLastError();
}

cudaError_t launch_prim_init(double* P, size_t plane, bool mag, int nblocks, cudaStream_t st) {
  if (mag)
    prim_init_kernel<true><<<nblocks, 256, 0, st>>>(P, plane);
  else
    prim_init_kernel<false><<<nblocks, 256, 0, st>>>(P, plane);
  return cudaGetLastError();
}

cudaError_t launch_prim_from_u(const double* U, double* P, size_t plane, bool mag, bool glm, int nblocks,
                               cudaStream_t st) {
  if (mag && glm)
    prim_from_u_kernel<true, true><<<nblocks, 256, 0, st>>>(U, P, plane);
  else if (mag)
    prim_from_u_kernel<true, false><<<nblocks, 256, 0, st>>>(U, P, plane);
  else
    prim_from_u_kernel<false, false><<<nblocks, 256, 0, st>>>(U, P, plane);
  return cudaGetLastError();
}

cudaError_t launch_prim_out(const double* P, size_t plane, double phifac, double gm1, double* out, double* p_out,
                            int nblocks, cudaStream_t st) {
  prim_out_kernel<<<nblocks, 256, 0, st>>>(P, plane, phifac, gm1, out, p_out);
  return cudaGetLastError();
}

// evo_output (output.f90:147-275): each block adds its cells' contributions
// to the ten totals (mass, total, internal and twice the kinetic energy,
// gravitational energy, bound mass, energy and angular momentum, twice the
// magnetic energy, angular momentum); evo_final_kernel adds the blocks'
// partials in block order, so the result does not depend on scheduling.
// dvol follows metric.f90 as the CFL reduction forms it.
constexpr int kEvoThreads = 256;

__global__ void __launch_bounds__(kEvoThreads) evo_kernel(const GridDev G, const double* P, size_t plane,
                                                         const double* gphi, const double* sinc, double* part) {
  __shared__ double red[kEvoQ][kEvoThreads];
  double acc[kEvoQ];
#pragma unroll
  for (int q = 0; q < kEvoQ; q++) acc[q] = 0.0;
  const int n0 = G.n[0], n1 = G.n[1];
  const SphGeo& M = G.sph;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < plane; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % n0), j = (int)((c / n0) % n1), k = (int)(c / ((size_t)n0 * n1));
    const double dxi1 = G.g[0].dxi[i + 2], dxi2 = G.g[1].dxi[j + 2], dxi3 = G.g[2].dxi[k + 2];
    double dvol;
    if (M.on && M.crd == 1)
      dvol = 0.5 * M.ar2[i + 2] * dxi2 * dxi3 * M.fac_j;
    else if (M.on)
      dvol = M.vr[i + 2] * M.cd[j + 2] * dxi3 * M.fac_j * M.fac_k;
    else
      dvol = dxi1 * dxi2 * dxi3;
    const double d = P[c], v1 = P[PV * plane + c], v2 = P[(PV + 1) * plane + c], v3 = P[(PV + 2) * plane + c];
    const double e = P[PE * plane + c], eint = P[PEINT * plane + c];
    const double b1 = P[PB * plane + c], b2 = P[(PB + 1) * plane + c], b3 = P[(PB + 2) * plane + c];
    acc[0] = acc[0] + d * dvol;
    acc[1] = acc[1] + e * dvol;
    acc[2] = acc[2] + eint * dvol;
    acc[3] = acc[3] + d * (v1 * v1 + v2 * v2 + v3 * v3) * dvol;
    acc[8] = acc[8] + (b1 * b1 + b2 * b2 + b3 * b3) * dvol;
    double jl = 0.0;
    if (M.on && M.crd == 1) jl = d * G.g[0].x[i + 2] * v2 * dvol;
    if (M.on && M.crd == 2 && sinc) jl = d * G.g[0].x[i + 2] * sinc[j + 2] * v3 * dvol;
    acc[9] = acc[9] + jl;
    if (gphi) {  // totphi = grvphi (no external potential on this path)
      const double ph = gphi[c], tot = ph;
      acc[4] = acc[4] + d * (tot - 0.5 * ph) * dvol;
      if (tot + (e - eint) / d <= 0.0) {
        acc[5] = acc[5] + d * dvol;
        acc[6] = acc[6] + (e + d * (tot - 0.5 * ph)) * dvol;
        acc[7] = acc[7] + jl;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kEvoQ; q++) red[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int h = kEvoThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
#pragma unroll
      for (int q = 0; q < kEvoQ; q++) red[q][threadIdx.x] = red[q][threadIdx.x] + red[q][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < kEvoQ) part[(size_t)blockIdx.x * kEvoQ + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void evo_final_kernel(const double* part, int nblocks, double* out) {
  const int q = threadIdx.x;
  if (q >= kEvoQ) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; b++) s = s + part[(size_t)b * kEvoQ + q];
  out[q] = s;
}

cudaError_t launch_evo(const GridDev& G, const double* P, size_t plane, const double* gphi, const double* sinc,
                       double* part, int nblocks, double* out, cudaStream_t st) {
  evo_kernel<<<nblocks, kEvoThreads, 0, st>>>(G, P, plane, gphi, sinc, part);
  evo_final_kernel<<<1, 32, 0, st>>>(part, nblocks, out);
  return cudaGetLastError();
}

cudaError_t launch_advance(DevScalars* sc, cudaStream_t st) {
  advance_kernel<<<1, 32, 0, st>>>(sc);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Batched step: many independent simulations of uneven sizes advance in one
// launch per phase.  Each CTA walks a persistent loop over a work list of
// (simulation, tile) items; every simulation keeps its own dt, ch and clock
// in its descriptor, so a batch step equals one hormone.f90 step per grid.

using T3D = Tile<8, 8, 8, 640, 1>;
using T3D4 = Tile<8, 8, 4, 384, 2>;
using T2D = Tile<16, 16, 1, 288, 3>;
using T2D8 = Tile<32, 8, 1, 320, 3>;
using T1D = Tile<256, 1, 1, 288, 3>;

// tile ids: 0 3-D 8x8x8 (640 threads), 1 3-D 8x8x4 (256 threads, 2 CTAs/SM),
// 2 2-D 16x16, 3 2-D 32x8, 4 1-D 256.  batch_tile_kind gives the grid's
// kind (0 3-D, 1 2-D x-y, 2 1-D x); each kind has the tile ids listed in
// batch_tile_variants.
int batch_tile_kind(const int solve[3]) {
  const int dim = solve[0] + solve[1] + solve[2];
  if (dim == 3) return 0;
  if (dim == 2 && solve[0] && solve[1]) return 1;
  if (dim == 1 && solve[0]) return 2;
  return -1;  // other orientations are run as single grids
}

int batch_tile_variants(int kind, int* ids) {
  if (kind == 0) {
    ids[0] = 0;
    ids[1] = 1;
    return 2;
  }
  if (kind == 1) {
    ids[0] = 2;
    ids[1] = 3;
    return 2;
  }
  ids[0] = 4;
  return 1;
}

void batch_tile_shape(int tid, int tile[3]) {
  const int shapes[5][3] = {{8, 8, 8}, {8, 8, 4}, {16, 16, 1}, {32, 8, 1}, {256, 1, 1}};
  for (int a = 0; a < 3; a++) tile[a] = shapes[tid][a];
}

template <bool MAG, bool GLM, class TL, bool DYN>
__global__ void __launch_bounds__(TL::NT, TL::MINB) batch_stage_kernel(SimDesc* sims, const int2* items, int nitems,
                                                                        int stage, int rk, int* queue) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SmemT<TL>& sm = *reinterpret_cast<SmemT<TL>*>(smem_raw);
  for_each_item<DYN>(nitems, queue, [&](int it) {
    const int2 w = items[it];
    SimDesc& S = sims[w.x];
    if (!S.active || S.sc.done) return;
    const StageArgs A = batch_stage_args(S, stage, rk);
    stage_tile_exact<MAG, GLM, TL>(S.G, A, sm, w.y, nullptr);
    __syncthreads();
  });
}

template <bool MAG, class TL>
__global__ void __launch_bounds__(TL::NT) batch_cfl_kernel(SimDesc* sims, const int2* items, int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    SimDesc& S = sims[w.x];
    if (!S.active || S.sc.done) continue;
    const GridDev& G = S.G;
    int bid = w.y, t0[3], T[3];
    constexpr int TT[3] = {TL::TX, TL::TY, TL::TZ};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int ti = bid % S.tiles[a];
      bid /= S.tiles[a];
      t0[a] = ti * TT[a];
      T[a] = min(TT[a], G.n[a] - t0[a]);
    }
    double my_dti = __longlong_as_double(0x7ff0000000000000LL), my_cf = 0.0;
    const double* P = S.P[S.pcur];
    for (int c = threadIdx.x; c < TL::NC; c += TL::NT) {
      const int cx = c % TL::TX, cy = (c / TL::TX) % TL::TY, cz = c / (TL::TX * TL::TY);
      if (cx >= T[0] || cy >= T[1] || cz >= T[2]) continue;
      const int i = t0[0] + cx, j = t0[1] + cy, k = t0[2] + cz;
      double dti, cfm;
      if (!cfl_cell<MAG>(G, P, S.plane, S.gamma, cidx(G, i, j, k), i, j, k, &S.sc, dti, cfm)) continue;
      my_cf = fmax2(my_cf, cfm);
      my_dti = fmin2(my_dti, dti);
    }
    cfl_block_reduce(my_dti, my_cf, &S.sc);
  }
}

__global__ void batch_finalize_kernel(SimDesc* sims, int nsims) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsims || !sims[s].active || sims[s].sc.done || sims[s].held) return;
  finalize_dt(&sims[s].sc);
}

// time += dt, tn += 1, end check (hormone.f90:147-155); primitive buffer
// parity and the phidamp factor (source.f90:239-260) for the next step
__global__ void batch_advance_kernel(SimDesc* sims, int nsims) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsims) return;
  SimDesc& S = sims[s];
  if (!S.active || S.sc.done || S.held) return;
  S.sc.time = S.sc.time + S.sc.dt;
  S.sc.tn = S.sc.tn + 1;
  S.pcur = (S.pcur + S.rktype) & 1;
  if (S.rktype == 1) {
    double* t = S.U[0];
    S.U[0] = S.U[1];
    S.U[1] = t;
  }
  S.phifac = S.glm ? S.damp : 1.0;
  if (S.sc.endstyle == 1 && S.sc.time >= S.sc.t_end) S.sc.done = 1;
}

// shared-memory opt-in of a batched stage kernel, done once (before any
// stream capture: rebuilding a batch's work list queries occupancy first)
template <bool MAG, bool GLM, class TL>
static cudaError_t batch_attr_t() {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(batch_stage_kernel<MAG, GLM, TL, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SmemT<TL>));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(batch_stage_kernel<MAG, GLM, TL, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(SmemT<TL>));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  return cudaSuccess;
}

template <bool MAG, bool GLM, class TL>
static cudaError_t launch_batch_stage_t(SimDesc* sims, const int2* items, int nitems, int stage, int rk, int grid,
                                        int* queue, cudaStream_t st) {
  cudaError_t e = batch_attr_t<MAG, GLM, TL>();
  if (e != cudaSuccess) return e;
  if (queue)
    batch_stage_kernel<MAG, GLM, TL, true>
        <<<grid, TL::NT, sizeof(SmemT<TL>), st>>>(sims, items, nitems, stage, rk, queue);
  else
    batch_stage_kernel<MAG, GLM, TL, false>
        <<<grid, TL::NT, sizeof(SmemT<TL>), st>>>(sims, items, nitems, stage, rk, nullptr);
  return cudaGetLastError();
}

template <class TL>
static cudaError_t launch_batch_stage_tl(SimDesc* sims, const int2* items, int nitems, bool mag, bool glm, int stage,
                                         int rk, int grid, int* queue, cudaStream_t st) {
  if (mag && glm) return launch_batch_stage_t<true, true, TL>(sims, items, nitems, stage, rk, grid, queue, st);
  if (mag) return launch_batch_stage_t<true, false, TL>(sims, items, nitems, stage, rk, grid, queue, st);
  return launch_batch_stage_t<false, false, TL>(sims, items, nitems, stage, rk, grid, queue, st);
}

cudaError_t launch_batch_stage(SimDesc* sims, const int2* items, int nitems, int tid, bool mag, bool glm, int stage,
                               int rk, int precision, int grid, int* queue, cudaStream_t st) {
  if (precision == 1)
    return launch_batch_stage_mixed(sims, items, nitems, tid, mag, glm, stage, rk, grid, queue, st);
  switch (tid) {
    case 0: return launch_batch_stage_tl<T3D>(sims, items, nitems, mag, glm, stage, rk, grid, queue, st);
    case 1: return launch_batch_stage_tl<T3D4>(sims, items, nitems, mag, glm, stage, rk, grid, queue, st);
    case 2: return launch_batch_stage_tl<T2D>(sims, items, nitems, mag, glm, stage, rk, grid, queue, st);
    case 3: return launch_batch_stage_tl<T2D8>(sims, items, nitems, mag, glm, stage, rk, grid, queue, st);
    case 4: return launch_batch_stage_tl<T1D>(sims, items, nitems, mag, glm, stage, rk, grid, queue, st);
  }
  return cudaErrorInvalidValue;
}

template <bool MAG, bool GLM, class TL>
static int occupancy_t() {
  int n = 0;
  batch_attr_t<MAG, GLM, TL>();
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_stage_kernel<MAG, GLM, TL, true>, TL::NT,
                                                sizeof(SmemT<TL>));  // the static split's shared memory is no larger
  return n > 0 ? n : 1;
}

template <class TL>
static int occupancy_tl(bool mag, bool glm) {
  if (mag && glm) return occupancy_t<true, true, TL>();
  if (mag) return occupancy_t<true, false, TL>();
  return occupancy_t<false, false, TL>();
}

int batch_stage_blocks_per_sm(int tid, bool mag, bool glm, int precision) {
  if (precision == 1) return batch_stage_mixed_blocks_per_sm(tid, mag, glm);
  switch (tid) {
    case 0: return occupancy_tl<T3D>(mag, glm);
    case 1: return occupancy_tl<T3D4>(mag, glm);
    case 2: return occupancy_tl<T2D>(mag, glm);
    case 3: return occupancy_tl<T2D8>(mag, glm);
  }
  return occupancy_tl<T1D>(mag, glm);
}

template <class TL>
static void batch_cfl_tl(SimDesc* sims, const int2* items, int nitems, bool mag, int grid, cudaStream_t st) {
  if (mag)
    batch_cfl_kernel<true, TL><<<grid, TL::NT, 0, st>>>(sims, items, nitems);
  else
    batch_cfl_kernel<false, TL><<<grid, TL::NT, 0, st>>>(sims, items, nitems);
}

cudaError_t launch_batch_cfl(SimDesc* sims, const int2* items, int nitems, int tid, bool mag, int grid,
                             cudaStream_t st) {
  switch (tid) {
    case 0: batch_cfl_tl<T3D>(sims, items, nitems, mag, grid, st); break;
    case 1: batch_cfl_tl<T3D4>(sims, items, nitems, mag, grid, st); break;
    case 2: batch_cfl_tl<T2D>(sims, items, nitems, mag, grid, st); break;
    case 3: batch_cfl_tl<T2D8>(sims, items, nitems, mag, grid, st); break;
    default: batch_cfl_tl<T1D>(sims, items, nitems, mag, grid, st); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_batch_finalize(SimDesc* sims, int nsims, cudaStream_t st) {
  batch_finalize_kernel<<<(nsims + 127) / 128, 128, 0, st>>>(sims, nsims);
  return cudaGetLastError();
}

cudaError_t launch_batch_advance(SimDesc* sims, int nsims, cudaStream_t st) {
  batch_advance_kernel<<<(nsims + 127) / 128, 128, 0, st>>>(sims, nsims);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Hyperbolic self-gravity (gravity_hyperbolic.f90:61-125, 230-280) with a
// Cartesian 7-point Laplacian: the counterpart of the 3-D spherical
// coefficients of gravity_hyperbolic.f90:385-406 with unit radial weights;
// each non-periodic face carries the Robin condition phi ~ 1/r folded into
// the centre coefficient as gravity_hyperbolic.f90:400-404 does.

__device__ __forceinline__ double rdist(const GridDev& G, int i, int j, int k) {
  const double x = G.g[0].x[i + 2], y = G.g[1].x[j + 2], z = G.g[2].x[k + 2];
  return sqrt(x * x + y * y + z * z);
}

// one thread per cell of an x row segment; rows by (blockIdx.y, blockIdx.z)
// = (j, k), so no index division
// The Laplacian numerator of a cell on a face of the grid (or of a slab):
// the Robin image phi ~ 1/r folded into the diagonal on a free face, the
// periodic neighbour, or the neighbouring slab's layer (hg_stage_kernel).
__device__ __forceinline__ double hg_boundary_lap(const GridDev& G, int i, int j, int k, size_t c, double c0,
                                                  const double cm[3], const double cp[3], const double* ph) {
  const int ijk[3] = {i, j, k};
  // a z neighbour in the neighbouring slab comes from its halo layer
    const bool hlo = k == 0 && G.ghalo[0] != nullptr, hhi = k == G.n[2] - 1 && G.ghalo[1] != nullptr;
    bool use_m[3] = {true, true, true}, use_p[3] = {true, true, true};
    size_t nbm[3], nbp[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int n = G.n[a];
      const bool per = G.bc[a][0][0] == 0;
      const bool hm = a == 2 && hlo, hp = a == 2 && hhi;
      int m[3] = {i, j, k}, p[3] = {i, j, k};
      m[a] = ijk[a] - 1;
      p[a] = ijk[a] + 1;
      if (per) {
        if (m[a] < 0) m[a] += n;
        if (p[a] >= n) p[a] -= n;
      } else {
        if (ijk[a] == n - 1 && !hp) {
          c0 = c0 + cp[a] * rdist(G, i, j, k) / rdist(G, p[0], p[1], p[2]);
          use_p[a] = false;
        }
        if (ijk[a] == 0 && !hm) {
          c0 = c0 + cm[a] * rdist(G, i, j, k) / rdist(G, m[0], m[1], m[2]);
          use_m[a] = false;
        }
      }
      nbm[a] = use_m[a] && !hm ? cidx(G, m[0], m[1], m[2]) : c;
      nbp[a] = use_p[a] && !hp ? cidx(G, p[0], p[1], p[2]) : c;
    }
    const size_t hc = (size_t)i + (size_t)G.n[0] * j;
    double lap = c0 * ph[c];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if (use_m[a]) lap = lap + cm[a] * (a == 2 && hlo ? G.ghalo[0][hc] : ph[nbm[a]]);
      if (use_p[a]) lap = lap + cp[a] * (a == 2 && hhi ? G.ghalo[1][hc] : ph[nbp[a]]);
    }
    return lap;
}

// 16 blocks of 128 threads per SM (32 registers): the stage is bound by the
// latency of its loads, and the full 64 warps hide more of it than the 36
// that 56 registers allow (0.8 % of the 192^3 polytrope step).
__global__ void __launch_bounds__(128, 16) hg_stage_kernel(const GridDev G, const HGArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i < G.n[0]) {
    const size_t c = cidx(G, i, j, k);
    const AxisGeo &gx = G.g[0], &gy = G.g[1], &gz = G.g[2];
    double c0, cm[3], cp[3], cn;
    if (A.uni) {  // every cell's weights are these (formed on the host in this order)
      c0 = A.uc0;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        cm[a] = A.ucm[a];
        cp[a] = A.ucp[a];
      }
      cn = A.ucn;
    } else {
    c0 = -((gx.idx[i + 2] + gx.idx[i + 3]) * gy.dxi[j + 2] * gz.dxi[k + 2] +
           (gy.idx[j + 2] + gy.idx[j + 3]) * gx.dxi[i + 2] * gz.dxi[k + 2] +
           (gz.idx[k + 2] + gz.idx[k + 3]) * gx.dxi[i + 2] * gy.dxi[j + 2]);
    // neighbour weights: area over centre spacing, each quotient corrected
    // from idx = RN(1/dx) where the host vouched for it (FastDiv), else
    // IEEE division -- the same bits either way
    const double ayz = gy.dxi[j + 2] * gz.dxi[k + 2], axz = gx.dxi[i + 2] * gz.dxi[k + 2];
    const double axy = gx.dxi[i + 2] * gy.dxi[j + 2];
    bool slow = !G.idx_rn;
    if (!slow) {
      cm[0] = div_rn(ayz, gx.dx[i + 2], gx.idx[i + 2], slow);
      cp[0] = div_rn(ayz, gx.dx[i + 3], gx.idx[i + 3], slow);
      cm[1] = div_rn(axz, gy.dx[j + 2], gy.idx[j + 2], slow);
      cp[1] = div_rn(axz, gy.dx[j + 3], gy.idx[j + 3], slow);
      cm[2] = div_rn(axy, gz.dx[k + 2], gz.idx[k + 2], slow);
      cp[2] = div_rn(axy, gz.dx[k + 3], gz.idx[k + 3], slow);
    }
    if (slow) {
      cm[0] = ayz / gx.dx[i + 2];
      cp[0] = ayz / gx.dx[i + 3];
      cm[1] = axz / gy.dx[j + 2];
      cp[1] = axz / gy.dx[j + 3];
      cm[2] = axy / gz.dx[k + 2];
      cp[2] = axy / gz.dx[k + 3];
    }
    cn = gx.dxi[i + 2] * gy.dxi[j + 2] * gz.dxi[k + 2];
    }
    const double* ph = A.phi_in;
    double lap;
    const size_t nx = (size_t)G.n[0], nxy = nx * (size_t)G.n[1];
    if (i > 0 && i < G.n[0] - 1 && j > 0 && j < G.n[1] - 1 && k > 0 && k < G.n[2] - 1) {
      // interior cell: every neighbour is a cell of this grid
      lap = c0 * ph[c];
      lap = lap + cm[0] * ph[c - 1];
      lap = lap + cp[0] * ph[c + 1];
      lap = lap + cm[1] * ph[c - nx];
      lap = lap + cp[1] * ph[c + nx];
      lap = lap + cm[2] * ph[c - nxy];
      lap = lap + cp[2] * ph[c + nxy];
    } else {
      lap = hg_boundary_lap(G, i, j, k, c, c0, cm, cp, ph);
    }
    double lapphi;
    if (A.uni && A.urcn_ok) {
      bool bad = false;
      lapphi = div_rn(lap, cn, A.urcn, bad);
      if (bad) lapphi = lap / cn;
    } else {
      FastDiv fd;
      lapphi = fd.div(lap, cn, fd.rec(cn));
      if (fd.bad) lapphi = lap / cn;
    }
    const double hgsrc = A.fourpiG * A.dens[c];
    double o1, o2;
    const double phi0 = ph[c], psi0 = A.psi_in[c];
    if (A.stage1) {
      o1 = phi0;
      o2 = psi0;
      A.org_phi[c] = o1;
      A.org_psi[c] = o2;
    } else {
      o1 = A.org_phi[c];
      o2 = A.org_psi[c];
    }
    const double pn = A.faco * o1 + A.facn * phi0 + A.fdc * psi0;
    double sn = A.faco * o2 + A.facn * psi0 + A.fdc * (lapphi - hgsrc);
    if (A.last) sn = sn * A.damp;
    A.phi_out[c] = pn;
    A.psi_out[c] = sn;
  }
}

cudaError_t launch_hg_stage(const GridDev& G, const HGArgs& A, int nblocks, cudaStream_t st) {
  (void)nblocks;
  const int bx = G.n[0] < 128 ? ((G.n[0] + 31) / 32) * 32 : 128;
  const dim3 grid((G.n[0] + bx - 1) / bx, G.n[1], G.n[2]);
  hg_stage_kernel<<<grid, bx, 0, st>>>(G, A);
  return cudaGetLastError();
}

// The same RK sub-stage on a spherical grid (get_lapphi_hgsrc,
// gravity_hyperbolic.f90:243-270): the coefficients of setup_grv_hyperbolic
// come precomputed per cell (A.lc); the neighbour beyond r = xi1s is the
// value the last boundary pass copied there (A.gin), the other neighbours
// beyond a non-periodic face carry zero weight, and phi is periodic.
__global__ void __launch_bounds__(128) hg_stage_sph_kernel(const GridDev G, const HGArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= G.n[0]) return;
  const int n0 = G.n[0], n1 = G.n[1], n2 = G.n[2];
  const size_t c = cidx(G, i, j, k), pl = A.plane;
  const double* ph = A.phi_in;
  const double* L = A.lc;
  double lap = L[c] * ph[c];
  lap = lap + L[pl + c] * (i > 0 ? ph[c - 1] : A.gin[j + (size_t)n1 * k]);
  lap = lap + L[2 * pl + c] * (i + 1 < n0 ? ph[c + 1] : ph[c]);
  if (n1 > 1) {
    lap = lap + L[3 * pl + c] * (j > 0 ? ph[cidx(G, i, j - 1, k)] : ph[c]);
    lap = lap + L[4 * pl + c] * (j + 1 < n1 ? ph[cidx(G, i, j + 1, k)] : ph[c]);
  }
  if (n2 > 1) {
    lap = lap + L[5 * pl + c] * ph[cidx(G, i, j, k > 0 ? k - 1 : n2 - 1)];
    lap = lap + L[6 * pl + c] * ph[cidx(G, i, j, k + 1 < n2 ? k + 1 : 0)];
  }
  const double lapphi = lap / L[7 * pl + c];
  const double hgsrc = A.fourpiG * A.dens[c];
  double o1, o2;
  const double phi0 = ph[c], psi0 = A.psi_in[c];
  if (A.stage1) {
    o1 = phi0;
    o2 = psi0;
    A.org_phi[c] = o1;
    A.org_psi[c] = o2;
  } else {
    o1 = A.org_phi[c];
    o2 = A.org_psi[c];
  }
  const double pn = A.faco * o1 + A.facn * phi0 + A.fdc * psi0;
  double sn = A.faco * o2 + A.facn * psi0 + A.fdc * (lapphi - hgsrc);
  if (A.last) sn = sn * A.damp;
  A.phi_out[c] = pn;
  A.psi_out[c] = sn;
}

cudaError_t launch_hg_stage_sph(const GridDev& G, const HGArgs& A, cudaStream_t st) {
  const int bx = G.n[0] < 128 ? ((G.n[0] + 31) / 32) * 32 : 128;
  const dim3 grid((G.n[0] + bx - 1) / bx, G.n[1], G.n[2]);
  hg_stage_sph_kernel<<<grid, bx, 0, st>>>(G, A);
  return cudaGetLastError();
}

}  // namespace hmn
