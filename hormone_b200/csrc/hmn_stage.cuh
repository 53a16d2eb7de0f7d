// hmn_stage.cuh -- the device code of one fused FP64 RK stage of a tile
// (slopes, HLLD faces, flux divergence, RK combination, source, primitive
// recovery) and of the CFL reduction, shared by the kernels of
// hmn_kernels.cu and the persistent small-grid loop of hmn_small.cu.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "hmn_div.cuh"
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
    // the slopes go straight to their shared-memory slots (rows of S)
    if (A.limiter == 1)
      slopes_to<MAG, 1, TL::NR>(&sm.P[0][rm], &sm.P[0][r], &sm.P[0][rp], g, cg, &sm.S[0][w], TL::NSB);
    else if (A.limiter == 2)
      slopes_to<MAG, 2, TL::NR>(&sm.P[0][rm], &sm.P[0][r], &sm.P[0][rp], g, cg, &sm.S[0][w], TL::NSB);
    else
      slopes_to<MAG, 0, TL::NR>(&sm.P[0][rm], &sm.P[0][r], &sm.P[0][rp], g, cg, &sm.S[0][w], TL::NSB);
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
    // the flux goes straight into its conserved slots of F (put_flux:
    // numflux.f90:186-198, 359-371, 531-543)
    if (!face_flux_fast<MAG, TL::NR>(&sm.P[0][rL], &sm.P[0][rR], &sm.S[0][sL], TL::NSB, &sm.S[0][sR], TL::NSB, dx1,
                                     dx2, cn, c1, c2, A.gamma, A.gm1, ch, &sm.F[0][w], TL::NFB)) {
      int gi[3] = {t0[0] + fx, t0[1] + fy, t0[2] + fz};
      gi[AX] = gL;
      record_error(A.sc, kENEG_EINT, gi[0], gi[1], gi[2]);  // numflux.f90:117 -> error_flux
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
        const double f0 = sm.F[ICNT][w];  // the mass flux this thread just wrote
        const double sg = fsign(0.5, f0);
        const double fix = 1.0 / (suml * (0.5 + sg) + sumr * (0.5 - sg));
#pragma unroll
        for (int n = 0; n < TL::SP; n++)
          if (n < A.nspc) sm.F[9 + n][w] = fix * f0 * (spl[n] * (0.5 + sg) + spr[n] * (0.5 - sg));
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
template <bool MAG>
__device__ __forceinline__ bool cfl_values(const GridDev& G, double gamma, double d, double eint, double v1, double v2,
                                           double v3, double b1, double b2, double b3, int i, int j, int k,
                                           DevScalars* sc, double& dti, double& cfm);

// CFLOUT: also fold dti and the signal speed of each new cell (dti_cell,
// the next step's CFL reduction) into *cdti (min) and *ccf (max).
template <bool MAG, bool GLM, class TL, bool SPH = false, bool PUSH = false, bool CFLOUT = false>
__device__ __forceinline__ void stage_tile_exact(const GridDev& G, const StageArgs& A, SmemT<TL>& sm, int tile_id,
                                                 const TmaMaps* tm, double* cdti = nullptr, double* ccf = nullptr) {
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
  if constexpr (CFLOUT) {
    double dti, cfm;
    if (cfl_values<MAG>(G, A.gamma, d, eint, v1, v2, v3, b1, b2, b3, i, j, k, A.sc, dti, cfm)) {
      *ccf = fmax2(*ccf, cfm);
      *cdti = fmin2(*cdti, dti);
    }
  }
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

// ---------------------------------------------------------------------------
// CFL timestep (timestep.f90:45-98, dti_cell :125-183)

__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

// dti and the largest signal speed of one cell (dti_cell, timestep.f90:125-183,
// eostype 0); false (and the error recorded) if eint <= 0 or d <= 0
template <bool MAG>
__device__ __forceinline__ bool cfl_values(const GridDev& G, double gamma, double d, double eint, double v1, double v2,
                                           double v3, double b1, double b2, double b3, int i, int j, int k,
                                           DevScalars* sc, double& dti, double& cfm) {
  const double gm1 = gamma - 1.0;
  const double off0 = G.solve[0] ? 1.0 : 0.0, off1 = G.solve[1] ? 1.0 : 0.0, off2 = G.solve[2] ? 1.0 : 0.0;
  if (eint <= 0.0 || d <= 0.0) {
    record_error(sc, kENEG_EINT, i, j, k);
    return false;
  }
  const double p = gm1 * eint;
  const double cs = sqrt(gamma * p / d);
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

// the same for cell c of the primitive planes P
template <bool MAG>
__device__ __forceinline__ bool cfl_cell(const GridDev& G, const double* P, size_t plane, double gamma, size_t c,
                                         int i, int j, int k, DevScalars* sc, double& dti, double& cfm) {
  const double d = P[c], eint = P[PEINT * plane + c];
  const double v1 = P[plane + c], v2 = P[2 * plane + c], v3 = P[3 * plane + c];
  double b1 = 0.0, b2 = 0.0, b3 = 0.0;
  if (MAG) {
    b1 = P[5 * plane + c];
    b2 = P[6 * plane + c];
    b3 = P[7 * plane + c];
  }
  return cfl_values<MAG>(G, gamma, d, eint, v1, v2, v3, b1, b2, b3, i, j, k, sc, dti, cfm);
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

}  // namespace hmn
