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
#include "hmn_tile.cuh"

namespace hmn {

template <class TL>
struct SmemT {
  double P[NQ + TL::SP][TL::NR];  // first: every TMA box destination in it is 128-byte aligned
  double S[NS + TL::SP][TL::NSB];
  double F[9 + TL::SP][TL::NFB];
  uint64_t bar;                   // completion barrier of the region's bulk copies
};

// One axis of the fused stage: slopes, face fluxes, flux divergence of the
// thread's own cell added to acc[].
template <int AX, bool MAG, bool GLM, class TL, bool SPH = false>
__device__ __forceinline__ void axis_pass(const GridDev& G, const StageArgs& A, SmemT<TL>& sm, const int t0[3],
                                          const int T[3], double acc[9], double accs[], double ch) {
  constexpr int TX = TL::TX, TY = TL::TY, TZ = TL::TZ;
  constexpr int SBX = TX + (AX == 0 ? 2 : 0), SBY = TY + (AX == 1 ? 2 : 0), SBZ = TZ + (AX == 2 ? 2 : 0);
  constexpr int FBX = TX + (AX == 0 ? 1 : 0), FBY = TY + (AX == 1 ? 1 : 0), FBZ = TZ + (AX == 2 ? 1 : 0);
  constexpr int NSB = SBX * SBY * SBZ, NFB = FBX * FBY * FBZ;
  constexpr int SSTR = AX == 0 ? 1 : (AX == 1 ? SBX : SBX * SBY);
  constexpr int FSTR = AX == 0 ? 1 : (AX == 1 ? FBX : FBX * FBY);
  constexpr int cn = AX, c1 = (AX + 1) % 3, c2 = (AX + 2) % 3;
  const AxisGeo& g = G.g[AX];
  const int tid = threadIdx.x;
  constexpr int nsl = MAG ? NS : S_B;

  // ---- limited slopes of the tile +-1 along AX -------------------------------
  for (int w = tid; w < NSB; w += TL::NT) {
    const int sx = w % SBX, sy = (w / SBX) % SBY, sz = w / (SBX * SBY);
    int lc[3] = {sx, sy, sz};
    lc[AX] -= 1;
    if (lc[AX] > T[AX] || lc[0] >= T[0] + (AX == 0) || lc[1] >= T[1] + (AX == 1) || lc[2] >= T[2] + (AX == 2))
      continue;  // outside a ragged tile
    int lm[3] = {lc[0], lc[1], lc[2]}, lp[3] = {lc[0], lc[1], lc[2]};
    lm[AX] -= 1;
    lp[AX] += 1;
    const int r = TL::pidx(lc[0], lc[1], lc[2]);
    const int rm = TL::pidx(lm[0], lm[1], lm[2]);
    const int rp = TL::pidx(lp[0], lp[1], lp[2]);
    const int cg = lc[AX] + t0[AX];  // global coordinate along AX
    double sl[NS];
    if (A.limiter == 1)
      slopes_of<MAG, 1, TL::NR>(&sm.P[0][rm], &sm.P[0][r], &sm.P[0][rp], g, cg, sl);
    else if (A.limiter == 2)
      slopes_of<MAG, 2, TL::NR>(&sm.P[0][rm], &sm.P[0][r], &sm.P[0][rp], g, cg, sl);
    else
      slopes_of<MAG, 0, TL::NR>(&sm.P[0][rm], &sm.P[0][r], &sm.P[0][rp], g, cg, sl);
    // passive-scalar slopes (interpolation.f90:135-141), not zeroed by the eint check
    if constexpr (TL::SP > 0) {
      for (int n = 0; n < A.nspc; n++) {
        double du = 0.0;
        if (A.limiter != 0) {
          const double u0 = sm.P[NQ + n][rm], u1 = sm.P[NQ + n][r], u2 = sm.P[NQ + n][rp];
          if (A.limiter == 1)
            du = lim_minmod(u0, u1, u2, g.idx[cg + 2], g.idx[cg + 3], g.isum[cg + 2]);
          else
            du = lim_mmc(u0, u1, u2, g.mcf[cg + 2], g.mcb[cg + 2], g.ga[cg + 2], g.gb[cg + 2]);
        }
        sm.S[NS + n][w] = du;
      }
    }
#pragma unroll
    for (int q = 0; q < nsl; q++) sm.S[q][w] = sl[q];
  }
  __syncthreads();

  // ---- HLLD fluxes on the T+1 faces along AX --------------------------------
  for (int w = tid; w < NFB; w += TL::NT) {
    const int fx = w % FBX, fy = (w / FBX) % FBY, fz = w / (FBX * FBY);
    int fc[3] = {fx, fy, fz};
    const int f = fc[AX];  // face between local cells f-1 and f
    if (f > T[AX] || fx >= T[0] + (AX == 0) || fy >= T[1] + (AX == 1) || fz >= T[2] + (AX == 2)) continue;
    int lL[3] = {fx, fy, fz};
    lL[AX] = f - 1;
    int lR[3] = {lL[0], lL[1], lL[2]};
    lR[AX] = f;
    const int rL = TL::pidx(lL[0], lL[1], lL[2]), rR = TL::pidx(lR[0], lR[1], lR[2]);
    const int sL = fx + SBX * (fy + SBY * fz);  // slope-box index of the left cell (coordinate f along AX)
    const int sR = sL + SSTR;
    const int gL = t0[AX] + f - 1;
    const double dx1 = g.hr[gL + 2];  // xi(i)-x(i)
    const double dx2 = g.hl[gL + 3];  // x(i+1)-xi(i)
    double fl[9];
    if (!face_flux_fast<MAG, TL::NR>(&sm.P[0][rL], &sm.P[0][rR], &sm.S[0][sL], TL::NSB, &sm.S[0][sR], TL::NSB, dx1,
                                     dx2, cn, c1, c2, A.gamma, A.gm1, ch, fl)) {
      int gi[3] = {t0[0] + fx, t0[1] + fy, t0[2] + fz};
      gi[AX] = gL;
      record_error(A.sc, kENEG_EINT, gi[0], gi[1], gi[2]);  // numflux.f90:117 -> error_flux
    }
    // rotate back into the conserved slots (numflux.f90:186-198, 359-371, 531-543)
    sm.F[ICNT][w] = fl[0];
    sm.F[IMO1 + cn][w] = fl[1];
    sm.F[IMO1 + c1][w] = fl[2];
    sm.F[IMO1 + c2][w] = fl[3];
    sm.F[IENE][w] = fl[4];
    if (MAG) {
      sm.F[IMG1 + cn][w] = fl[5];
      sm.F[IMG1 + c1][w] = fl[6];
      sm.F[IMG1 + c2][w] = fl[7];
      if (GLM) sm.F[I9WV][w] = fl[8];
    }
    // boundary code 10: the inner z face carries the host's flux
    // (numflux.f90:566 -> fluxboundary.f90:42-87)
    if (AX == 2 && G.fb != nullptr && t0[2] + f == 0) {
#pragma unroll
      for (int q = 0; q < 9; q++) sm.F[q][w] = G.fb[q];
      if constexpr (TL::SP > 0)
        for (int n = 0; n < A.nspc; n++) sm.F[9 + n][w] = G.fb[9 + n];
      continue;
    }
    // passive scalars: face fractions upwinded by the mass flux and
    // renormalised to sum 1 (numflux.f90:200-212)
    if constexpr (TL::SP > 0) {
      if (A.nspc > 0) {
        double spl[TL::SP], spr[TL::SP];
        double suml = 0.0, sumr = 0.0;
#pragma unroll
        for (int n = 0; n < TL::SP; n++) {
          if (n < A.nspc) {
            spl[n] = sm.P[NQ + n][rL] + dx1 * sm.S[NS + n][sL];
            spr[n] = sm.P[NQ + n][rR] - dx2 * sm.S[NS + n][sR];
            suml = suml + spl[n];
            sumr = sumr + spr[n];
          }
        }
        const double sg = fsign(0.5, fl[0]);
        const double fix = 1.0 / (suml * (0.5 + sg) + sumr * (0.5 - sg));
#pragma unroll
        for (int n = 0; n < TL::SP; n++)
          if (n < A.nspc) sm.F[9 + n][w] = fix * fl[0] * (spl[n] * (0.5 + sg) + spr[n] * (0.5 - sg));
      }
    }
  }
  __syncthreads();

  // ---- flux divergence of the thread's own cell -------------------------------
  if (tid < TL::NC) {
    const int cx = tid % TX, cy = (tid / TX) % TY, cz = tid / (TX * TY);
    const int cc[3] = {cx, cy, cz};
    if (cx < T[0] && cy < T[1] && cz < T[2]) {
      const int wm = cx + FBX * (cy + FBY * cz);  // face on the low side
      const int wp = wm + FSTR;
      constexpr int nv = MAG ? (GLM ? 9 : 8) : 5;
      if constexpr (SPH) {
        double cw, fm, fp;
        sph_div_weights<AX>(G, cx + t0[0], cy + t0[1], cz + t0[2], cw, fm, fp);
#pragma unroll
        for (int q = 0; q < nv; q++) acc[q] = acc[q] + cw * (fm * sm.F[q][wm] - fp * sm.F[q][wp]);
      } else {
        const double idxi = g.idxi[cc[AX] + t0[AX] + 2];
#pragma unroll
        for (int q = 0; q < nv; q++) acc[q] = acc[q] + idxi * (sm.F[q][wm] - sm.F[q][wp]);
      }
      if constexpr (TL::SP > 0 && !SPH) {
        const double idxi = g.idxi[cc[AX] + t0[AX] + 2];
#pragma unroll
        for (int n = 0; n < TL::SP; n++)
          if (n < A.nspc) accs[n] = accs[n] + idxi * (sm.F[9 + n][wm] - sm.F[9 + n][wp]);
      }
    }
  }
  // S and F are reused by the next axis.  The barrier is not needed for
  // correctness (the next slope phase writes only S, and its own barrier
  // orders these reads of F before F is rewritten), but without it the FP64
  // stage is scheduled worse: 11.7 against 10.5 ms at 256^3.
  __syncthreads();
}

// One tile of one RK stage; `tile_id` enumerates the tiles of the grid
// (x fastest).  Shared by the single-grid and the batched kernels.
template <bool MAG, bool GLM, class TL, bool SPH = false, bool PUSH = false>
__device__ __forceinline__ void stage_tile_exact(const GridDev& G, const StageArgs& A, SmemT<TL>& sm, int tile_id,
                                                 const TmaMaps* tm) {
  const int tid = threadIdx.x;

  int bid = tile_id;
  int t0[3], T[3];
  constexpr int TT[3] = {TL::TX, TL::TY, TL::TZ};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int ti = bid % A.tiles[a];
    bid /= A.tiles[a];
    t0[a] = ti * TT[a];
    T[a] = min(TT[a], G.n[a] - t0[a]);
  }

  // ---- 1. stage the cross-shaped region --------------------------------------
  // Every slot of the full-tile layout is one local cell (pidx and
  // region_cell are inverse); a ragged tile needs the cells within two of
  // its real extent, so its high halo occupies interior-layout slots.
  stage_region<MAG, GLM, TL>(G, A, sm.P, &sm.bar, tm, t0, T);

  double acc[9];
#pragma unroll
  for (int q = 0; q < 9; q++) acc[q] = 0.0;
  double accs[TL::SP > 0 ? TL::SP : 1];
#pragma unroll
  for (int n = 0; n < (TL::SP > 0 ? TL::SP : 1); n++) accs[n] = 0.0;
  const double ch = A.sc->ch;
  if (TL::TX > 1 && G.solve[0]) axis_pass<0, MAG, GLM, TL, SPH>(G, A, sm, t0, T, acc, accs, ch);
  if (TL::TY > 1 && G.solve[1]) axis_pass<1, MAG, GLM, TL, SPH>(G, A, sm, t0, T, acc, accs, ch);
  if (TL::TZ > 1 && G.solve[2]) axis_pass<2, MAG, GLM, TL, SPH>(G, A, sm, t0, T, acc, accs, ch);

  // ---- RK combination (rungekutta.f90:35-59) + source (source.f90:70-85) -------
  if (tid >= TL::NC) return;
  const int cx = tid % TL::TX, cy = (tid / TL::TX) % TL::TY, cz = tid / (TL::TX * TL::TY);
  if (cx >= T[0] || cy >= T[1] || cz >= T[2]) return;
  const int i = t0[0] + cx, j = t0[1] + cy, k = t0[2] + cz;
  const size_t c = cidx(G, i, j, k);
  const size_t pl = A.plane;
  constexpr int nv = MAG ? (GLM ? 9 : 8) : 5;
  if constexpr (SPH) {
    // geometric sources and, with self-gravity, the force of the potential
    // with the spherical ghost images (source.f90:113-150), all in FP64
    double frc[3];
    if (A.gphi != nullptr) gravity_force<true>(G, A.gphi, c, i, j, k, A.pin[c], frc);
    sph_sources<MAG>(G, A, c, i, j, acc, A.gphi != nullptr ? frc : nullptr);
  } else {
    if (A.gphi != nullptr) {
      const double d = A.pin[c];
      const double v[3] = {A.pin[PV * pl + c], A.pin[(PV + 1) * pl + c], A.pin[(PV + 2) * pl + c]};
      double frc[3];
      const int ijk[3] = {i, j, k};
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const AxisGeo& g = G.g[a];
        const int s = ijk[a];
        // neighbours of the potential with the ghost images of the boundary
        // (periodic copy, or the Robin image phi ~ 1/r)
        double ph[3];
#pragma unroll
        for (int o = -1; o <= 1; o++) {
          int nb[3] = {i, j, k};
          nb[a] = s + o;
          if (nb[a] >= 0 && nb[a] < G.n[a]) {
            ph[o + 1] = A.gphi[cidx(G, nb[0], nb[1], nb[2])];
          } else if (a == 2 && G.ghalo[o > 0] != nullptr) {  // the neighbouring slab's layer
            ph[o + 1] = G.ghalo[o > 0][(size_t)i + (size_t)G.n[0] * j];
          } else if (G.bc[a][0][0] == 0) {
            nb[a] = nb[a] < 0 ? G.n[a] - 1 : 0;
            ph[o + 1] = A.gphi[cidx(G, nb[0], nb[1], nb[2])];
          } else {
            const double xe = G.g[0].x[i + 2], ye = G.g[1].x[j + 2], ze = G.g[2].x[k + 2];
            const double xg = G.g[0].x[nb[0] + 2], yg = G.g[1].x[nb[1] + 2], zg = G.g[2].x[nb[2] + 2];
            const double re = sqrt(xe * xe + ye * ye + ze * ze), rg = sqrt(xg * xg + yg * yg + zg * zg);
            ph[o + 1] = A.gphi[c] * re / rg;
          }
        }
        const double dxm = g.dx[s + 2], dxp = g.dx[s + 3], im = g.idx[s + 2], ip = g.idx[s + 3];
        frc[a] = -((dxm * ip * ph[2] - dxp * im * ph[0]) / (dxm + dxp) + (dxp - dxm) * im * ip * ph[1]) * d;
      }
      acc[1] = acc[1] + frc[0];
      acc[2] = acc[2] + frc[1];
      acc[3] = acc[3] + frc[2];
      acc[4] = acc[4] + (frc[0] * v[0] + frc[1] * v[1] + frc[2] * v[2]);
    }
  }
  const double dtf = A.fact * A.sc->dt;
  double un[9];
#pragma unroll
  for (int q = 0; q < nv; q++) {
    const double val = A.faco * A.uorg[q * pl + c] + A.facn * A.ucur[q * pl + c] + dtf * acc[q];
    un[q] = val;
    A.uout[q * pl + c] = val;
  }
  // primitive + pressure of the new state (rungekutta.f90:205-229, eos.f90:805-842)
  const double d = un[0];
  double v1, v2, v3;
  {
    FastDiv fd;
    const double rd = fd.rec(d);
    v1 = fd.div(un[1], d, rd);
    v2 = fd.div(un[2], d, rd);
    v3 = fd.div(un[3], d, rd);
    if (fd.bad) {
      v1 = un[1] / d;
      v2 = un[2] / d;
      v3 = un[3] / d;
    }
  }
  const double b1 = MAG ? un[5] : 0.0, b2 = MAG ? un[6] : 0.0, b3 = MAG ? un[7] : 0.0;
  const double eint = get_eint<MAG>(un[4], d, v1, v2, v3, b1, b2, b3);
  double* Po = A.pout;
  Po[c] = d;
  Po[PV * pl + c] = v1;
  Po[(PV + 1) * pl + c] = v2;
  Po[(PV + 2) * pl + c] = v3;
  Po[PE * pl + c] = un[4];
  Po[PB * pl + c] = b1;
  Po[(PB + 1) * pl + c] = b2;
  Po[(PB + 2) * pl + c] = b3;
  Po[PPHI * pl + c] = GLM ? un[8] : 0.0;
  Po[PEINT * pl + c] = eint;
  if (eint <= 0.0) record_error(A.sc, kENEG_EINT, i, j, k);
  // passive scalars from the new density (rungekutta.f90:61-86)
  if constexpr (TL::SP > 0) {
#pragma unroll
    for (int n = 0; n < TL::SP; n++) {
      if (n >= A.nspc) break;
      const double x = A.pin[(size_t)(NP + n) * pl + c];
      double xo;
      if (A.stage == 1) {
        xo = x * A.uorg[c];
        A.spcorg[(size_t)n * pl + c] = xo;
      } else {
        xo = A.spcorg[(size_t)n * pl + c];
      }
      Po[(size_t)(NP + n) * pl + c] = (A.faco * xo + A.facn * x * A.pin[c] + dtf * accs[n]) / d;
    }
  }
  if constexpr (PUSH) push_boundary_layers(G, A, Po, c, i, j, k);
}

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

// ---------------------------------------------------------------------------
// CFL timestep (timestep.f90:45-98, dti_cell :125-183)

__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

// dti and the largest signal speed of one cell (dti_cell, timestep.f90:125-183,
// eostype 0); false (and the error recorded) if eint <= 0 or d <= 0
template <bool MAG>
__device__ __forceinline__ bool cfl_cell(const GridDev& G, const double* P, size_t plane, double gamma, size_t c,
                                         int i, int j, int k, DevScalars* sc, double& dti, double& cfm) {
  const double gm1 = gamma - 1.0;
  const double off0 = G.solve[0] ? 1.0 : 0.0, off1 = G.solve[1] ? 1.0 : 0.0, off2 = G.solve[2] ? 1.0 : 0.0;
  const double d = P[c], eint = P[PEINT * plane + c];
  const double v1 = P[plane + c], v2 = P[2 * plane + c], v3 = P[3 * plane + c];
  if (eint <= 0.0 || d <= 0.0) {
    record_error(sc, kENEG_EINT, i, j, k);
    return false;
  }
  const double p = gm1 * eint;
  const double cs = sqrt(gamma * p / d);
  double cf1, cf2, cf3;
  if (MAG) {
    const double b1 = P[5 * plane + c], b2 = P[6 * plane + c], b3 = P[7 * plane + c];
    cf1 = get_cf(d, cs, b1, b2, b3) + fabs(v1);
    cf2 = get_cf(d, cs, b2, b1, b3) + fabs(v2);
    cf3 = get_cf(d, cs, b3, b1, b2) + fabs(v3);
  } else {
    cf1 = cs + fabs(v1);
    cf2 = cs + fabs(v2);
    cf3 = cs + fabs(v3);
  }
  const double dxi1 = G.g[0].dxi[i + 2], dxi2 = G.g[1].dxi[j + 2], dxi3 = G.g[2].dxi[k + 2];
  if (G.sph.on && G.sph.crd == 1) {  // metric.f90:80-96, one phi cell: dvol, sa1, sa3 times four
    const SphGeo& M = G.sph;
    const double ar = M.ar2[i + 2], f4 = M.fac_j;
    const double dvol = 0.5 * ar * dxi2 * dxi3 * f4;
    const double sa1m = M.detg1[i + 1] * dxi2 * dxi3 * f4, sa1p = M.detg1[i + 2] * dxi2 * dxi3 * f4;
    const double sa2 = dxi1 * dxi3, sa3 = 0.5 * ar * dxi2 * f4;
    dti = dvol / (cf1 * off0 * (sa1m + sa1p) + cf2 * off1 * (sa2 + sa2) + cf3 * off2 * (sa3 + sa3));
  } else if (G.sph.on) {  // metric.f90:117-130
    const SphGeo& M = G.sph;
    const double cd = M.cd[j + 2], fj = M.fac_j, fk = M.fac_k, ar = M.ar2[i + 2];
    const double dvol = M.vr[i + 2] * cd * dxi3 * fj * fk;
    const double sa1m = M.hr2[i + 1] * cd * dxi3 * fj * fk, sa1p = M.hr2[i + 2] * cd * dxi3 * fj * fk;
    const double sa2m = 0.5 * M.sini[j + 1] * ar * dxi3 * fk, sa2p = 0.5 * M.sini[j + 2] * ar * dxi3 * fk;
    const double sa3 = 0.5 * ar * dxi2 * fj;
    dti = dvol / (cf1 * off0 * (sa1m + sa1p) + cf2 * off1 * (sa2m + sa2p) + cf3 * off2 * (sa3 + sa3));
  } else {
    const double dvol = dxi1 * dxi2 * dxi3;  // metric.f90:45-48
    const double sa1 = dxi2 * dxi3, sa2 = dxi1 * dxi3, sa3 = dxi1 * dxi2;
    dti = dvol / (cf1 * off0 * (sa1 + sa1) + cf2 * off1 * (sa2 + sa2) + cf3 * off2 * (sa3 + sa3));
  }
  cfm = fmax2(fmax2(cf1, cf2), cf3);
  return true;
}

// block-wide min(dti), max(cf) folded into the simulation's reduction slots
__device__ __forceinline__ void cfl_block_reduce(double my_dti, double my_cf, DevScalars* sc) {
  for (int o = 16; o > 0; o >>= 1) {
    my_dti = fmin2(my_dti, __shfl_xor_sync(0xffffffffu, my_dti, o));
    my_cf = fmax2(my_cf, __shfl_xor_sync(0xffffffffu, my_cf, o));
  }
  __shared__ double rd[32], rc[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    rd[wid] = my_dti;
    rc[wid] = my_cf;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    my_dti = lane < nw ? rd[lane] : __longlong_as_double(0x7ff0000000000000LL);
    my_cf = lane < nw ? rc[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      my_dti = fmin2(my_dti, __shfl_xor_sync(0xffffffffu, my_dti, o));
      my_cf = fmax2(my_cf, __shfl_xor_sync(0xffffffffu, my_cf, o));
    }
    if (lane == 0) {
      atomicMin(&sc->min_dti_bits, (unsigned long long)__double_as_longlong(my_dti));
      atomicMax(&sc->cfmax_bits, (unsigned long long)__double_as_longlong(my_cf));
    }
  }
  __syncthreads();
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


// dt from the reduced values, with the output/end-time clamps
// (timestep.f90:74-98).  One thread; also re-arms the reduction slots.
__device__ __forceinline__ void finalize_dt(DevScalars* sc) {
  const double mind = __longlong_as_double((long long)sc->min_dti_bits);
  const double cfmax = __longlong_as_double((long long)sc->cfmax_bits);
  double dt = sc->courant * mind;
  const double time = sc->time, t_out = sc->t_out, t_end = sc->t_end;
  if (sc->outstyle == 1) {
    double t_ref = t_out;
    if (sc->endstyle == 1) t_ref = fmin2(t_out, t_end);
    if (t_ref - time - dt > 0.0 && t_ref - time - 2.0 * dt < 0.0)
      dt = 0.5 * (t_ref - time);
    else
      dt = fmin2(dt, t_out - time);
  }
  if (sc->endstyle == 1) dt = fmin2(dt, t_end - time);
  sc->dt = dt;
  sc->ch = cfmax;
  sc->cfmax = cfmax;
  if (sc->gravswitch == 3) {
    double cg = sc->HGfac * cfmax;
    if (sc->maxtngrv > 0) cg = fmin2(cg, sc->hgcfl * sc->dtg_unit * (double)sc->maxtngrv / dt);
    sc->cgrav = cg;
    sc->dtgrav = fmin2(dt, sc->hgcfl * sc->dtg_unit / cg);
  }
  sc->min_dti_bits = 0x7ff0000000000000ULL;
  sc->cfmax_bits = 0ULL;
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
void stage_tile(const int solve[3], int precision, int nspc, int tile[3]) {
  const int dim = solve[0] + solve[1] + solve[2];
  for (int a = 0; a < 3; a++) tile[a] = 1;
  if (dim == 3 && nspc > 0) {  // the scalar planes only fit the smaller tile
    tile[0] = 8;
    tile[1] = 8;
    tile[2] = 4;
  } else if (dim == 3) {
    const char* env = getenv("HMN_TILE3D");
    bool t884 = precision == 1;
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
  if (t[0] == 16 && t[1] == 16 && t[2] == 1) return launch_stage_tl<Tile<16, 16, 1, 288, 2>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 16 && t[1] == 1 && t[2] == 16) return launch_stage_tl<Tile<16, 1, 16, 288, 2>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 16 && t[2] == 16) return launch_stage_tl<Tile<1, 16, 16, 288, 2>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 256 && t[1] == 1 && t[2] == 1) return launch_stage_tl<Tile<256, 1, 1, 288, 2>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 256 && t[2] == 1) return launch_stage_tl<Tile<1, 256, 1, 288, 2>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 1 && t[2] == 256) return launch_stage_tl<Tile<1, 1, 256, 288, 2>>(G, A, mag, glm, nullptr, st);
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
using T2D = Tile<16, 16, 1, 288, 2>;
using T2D8 = Tile<32, 8, 1, 320, 2>;
using T1D = Tile<256, 1, 1, 288, 2>;

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

template <bool MAG, bool GLM, class TL>
__global__ void __launch_bounds__(TL::NT, TL::MINB) batch_stage_kernel(SimDesc* sims, const int2* items, int nitems,
                                                                        int stage, int rk) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SmemT<TL>& sm = *reinterpret_cast<SmemT<TL>*>(smem_raw);
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 w = items[it];
    SimDesc& S = sims[w.x];
    if (!S.active || S.sc.done) continue;
    const StageArgs A = batch_stage_args(S, stage, rk);
    stage_tile_exact<MAG, GLM, TL>(S.G, A, sm, w.y, nullptr);
    __syncthreads();
  }
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
    cudaError_t e = cudaFuncSetAttribute(batch_stage_kernel<MAG, GLM, TL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SmemT<TL>));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  return cudaSuccess;
}

template <bool MAG, bool GLM, class TL>
static cudaError_t launch_batch_stage_t(SimDesc* sims, const int2* items, int nitems, int stage, int rk, int grid,
                                        cudaStream_t st) {
  cudaError_t e = batch_attr_t<MAG, GLM, TL>();
  if (e != cudaSuccess) return e;
  batch_stage_kernel<MAG, GLM, TL><<<grid, TL::NT, sizeof(SmemT<TL>), st>>>(sims, items, nitems, stage, rk);
  return cudaGetLastError();
}

template <class TL>
static cudaError_t launch_batch_stage_tl(SimDesc* sims, const int2* items, int nitems, bool mag, bool glm, int stage,
                                         int rk, int grid, cudaStream_t st) {
  if (mag && glm) return launch_batch_stage_t<true, true, TL>(sims, items, nitems, stage, rk, grid, st);
  if (mag) return launch_batch_stage_t<true, false, TL>(sims, items, nitems, stage, rk, grid, st);
  return launch_batch_stage_t<false, false, TL>(sims, items, nitems, stage, rk, grid, st);
}

cudaError_t launch_batch_stage(SimDesc* sims, const int2* items, int nitems, int tid, bool mag, bool glm, int stage,
                               int rk, int precision, int grid, cudaStream_t st) {
  if (precision == 1) return launch_batch_stage_mixed(sims, items, nitems, tid, mag, glm, stage, rk, grid, st);
  switch (tid) {
    case 0: return launch_batch_stage_tl<T3D>(sims, items, nitems, mag, glm, stage, rk, grid, st);
    case 1: return launch_batch_stage_tl<T3D4>(sims, items, nitems, mag, glm, stage, rk, grid, st);
    case 2: return launch_batch_stage_tl<T2D>(sims, items, nitems, mag, glm, stage, rk, grid, st);
    case 3: return launch_batch_stage_tl<T2D8>(sims, items, nitems, mag, glm, stage, rk, grid, st);
    case 4: return launch_batch_stage_tl<T1D>(sims, items, nitems, mag, glm, stage, rk, grid, st);
  }
  return cudaErrorInvalidValue;
}

template <bool MAG, bool GLM, class TL>
static int occupancy_t() {
  int n = 0;
  batch_attr_t<MAG, GLM, TL>();
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_stage_kernel<MAG, GLM, TL>, TL::NT, sizeof(SmemT<TL>));
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

__global__ void __launch_bounds__(128) hg_stage_kernel(const GridDev G, const HGArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i < G.n[0]) {
    const size_t c = cidx(G, i, j, k);
    const AxisGeo &gx = G.g[0], &gy = G.g[1], &gz = G.g[2];
    double c0 = -((gx.idx[i + 2] + gx.idx[i + 3]) * gy.dxi[j + 2] * gz.dxi[k + 2] +
                  (gy.idx[j + 2] + gy.idx[j + 3]) * gx.dxi[i + 2] * gz.dxi[k + 2] +
                  (gz.idx[k + 2] + gz.idx[k + 3]) * gx.dxi[i + 2] * gy.dxi[j + 2]);
    double cm[3], cp[3];
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
    const double cn = gx.dxi[i + 2] * gy.dxi[j + 2] * gz.dxi[k + 2];
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
    {
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
