// hmn_mixed.cu -- the mixed-precision form of the fused RK stage.
//
// Same tile structure, boundary images and step semantics as the FP64
// stage_kernel (hmn_kernels.cu), with the arithmetic split by what needs
// double precision:
//   * reconstruction in FP64, with the limiters' divisions by grid spacings
//     replaced by products with precomputed reciprocals, and the FP64
//     reciprocals of densities by two Newton-Raphson steps from the
//     approximate reciprocal (within about one ulp, no branch);
//   * pressure recovery eint = E - kinetic - magnetic in FP64, in the cells
//     and on both sides of every face (high Mach / low beta cancellation);
//   * the HLLD Riemann solver, the EOS and the fast speeds in FP32
//     (approximate reciprocal and square root: this translation unit is
//     compiled with -use_fast_math, which only affects single precision);
//   * slopes and fluxes kept in shared memory as FP32;
//   * the flux divergence and the RK combination in FP64, the three terms of
//     faco*U^n + facn*U^s + fact*dt*L summed with compensated (TwoSum)
//     additions.
// The result is not bit-compatible with the reference; its error against the
// FP64 path is measured (L1 per variable) by the tests and the benchmark.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "hmn_div.cuh"
#include "hmn_internal.h"
#include "hmn_math.cuh"
#include "hmn_queue.cuh"
#include "hmn_tile.cuh"

namespace hmn {

template <class TL>
struct SmemMixed {
  double P[NQ][TL::NR];  // first: every TMA box destination in it is 128-byte aligned
  float S[NS][TL::NSB];
  float F[9][TL::NFB];
  uint64_t bar;          // completion barrier of the region's bulk copies
};

// s + e == a + b exactly (Knuth's TwoSum); intrinsics keep every operation
// separately rounded.
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

__device__ __forceinline__ double mmc_fast(double u0, double u1, double u2, double cf, double cb, double gab,
                                           double rga) {
  const double top = (u1 - u0) * gab;
  const double bot = u2 - u1;
  const double sig = fsign(1.0, bot);
  double m = sig * 0.5 * (bot + top);
  m = fmin2(m, sig * cf * bot);
  m = fmin2(m, sig * cb * top);
  return sig * fmax2(0.0, m) * rga;
}

__device__ __forceinline__ double minmod_fast(double u0, double u1, double u2, double i0, double i1, double risum) {
  const double x = 1.4 * (u2 - u1) * i1;
  const double y = 1.4 * (u1 - u0) * i0;
  const double z = (u2 - u0) * i0 * i1 * risum;
  const double s = fsign(1.0, x);
  double m = fabs(x);
  m = fmin2(m, s * y);
  m = fmin2(m, s * z);
  return s * fmax2(0.0, m);
}

template <int AX, bool MAG, bool GLM, class TL, bool SPH = false>
__device__ __forceinline__ void axis_pass_mixed(const GridDev& G, const StageArgs& A, SmemMixed<TL>& sm,
                                                const int t0[3], const int T[3], double acc[9], float ch) {
  constexpr int TX = TL::TX, TY = TL::TY, TZ = TL::TZ;
  constexpr int SBX = TX + (AX == 0 ? 2 : 0), SBY = TY + (AX == 1 ? 2 : 0), SBZ = TZ + (AX == 2 ? 2 : 0);
  constexpr int FBX = TX + (AX == 0 ? 1 : 0), FBY = TY + (AX == 1 ? 1 : 0), FBZ = TZ + (AX == 2 ? 1 : 0);
  constexpr int NSB = SBX * SBY * SBZ, NFB = FBX * FBY * FBZ;
  constexpr int SSTR = AX == 0 ? 1 : (AX == 1 ? SBX : SBX * SBY);
  constexpr int FSTR = AX == 0 ? 1 : (AX == 1 ? FBX : FBX * FBY);
  constexpr int cn = AX, c1 = (AX + 1) % 3, c2 = (AX + 2) % 3;
  constexpr int nsl = MAG ? NS : S_B;
  const AxisGeo& g = G.g[AX];
  const int tid = threadIdx.x;

  for (int w = tid; w < NSB; w += TL::NT) {
    const int sx = w % SBX, sy = (w / SBX) % SBY, sz = w / (SBX * SBY);
    int lc[3] = {sx, sy, sz};
    lc[AX] -= 1;
    if (lc[AX] > T[AX] || lc[0] >= T[0] + (AX == 0) || lc[1] >= T[1] + (AX == 1) || lc[2] >= T[2] + (AX == 2))
      continue;
    int lm[3] = {lc[0], lc[1], lc[2]}, lp[3] = {lc[0], lc[1], lc[2]};
    lm[AX] -= 1;
    lp[AX] += 1;
    const int r = TL::pidx(lc[0], lc[1], lc[2]);
    const int rm = TL::pidx(lm[0], lm[1], lm[2]);
    const int rp = TL::pidx(lp[0], lp[1], lp[2]);
    const int cg = lc[AX] + t0[AX];
    double sl[NS];
#pragma unroll
    for (int q = 0; q < NS; q++) sl[q] = 0.0;
    if (A.limiter != 0) {
      constexpr int qmap[NS] = {Q_D, Q_E, Q_M + 0, Q_M + 1, Q_M + 2, Q_B + 0, Q_B + 1, Q_B + 2};
      const double hl = g.hl[cg + 2], hr = g.hr[cg + 2];
      double L[NS], R[NS];
      if (A.limiter == 1) {
        const double i0 = g.idx[cg + 2], i1 = g.idx[cg + 3], ris = g.risum[cg + 2];
#pragma unroll
        for (int q = 0; q < nsl; q++) {
          const double u0 = sm.P[qmap[q]][rm], u1 = sm.P[qmap[q]][r], u2 = sm.P[qmap[q]][rp];
          const double du = minmod_fast(u0, u1, u2, i0, i1, ris);
          sl[q] = du;
          L[q] = u1 - hl * du;
          R[q] = u1 + hr * du;
        }
      } else {
        const double cf = g.mcf[cg + 2], cb = g.mcb[cg + 2], gab = g.gab[cg + 2], rga = g.rga[cg + 2];
#pragma unroll
        for (int q = 0; q < nsl; q++) {
          const double u0 = sm.P[qmap[q]][rm], u1 = sm.P[qmap[q]][r], u2 = sm.P[qmap[q]][rp];
          const double du = mmc_fast(u0, u1, u2, cf, cb, gab, rga);
          sl[q] = du;
          L[q] = u1 - hl * du;
          R[q] = u1 + hr * du;
        }
      }
      const double rdl = rcp_nr(L[S_D]), rdr = rcp_nr(R[S_D]);
      double eintl = L[S_E] - 0.5 * (L[S_M] * L[S_M] + L[S_M + 1] * L[S_M + 1] + L[S_M + 2] * L[S_M + 2]) * rdl;
      double eintr = R[S_E] - 0.5 * (R[S_M] * R[S_M] + R[S_M + 1] * R[S_M + 1] + R[S_M + 2] * R[S_M + 2]) * rdr;
      if (MAG) {
        eintl = eintl - 0.5 * (L[S_B] * L[S_B] + L[S_B + 1] * L[S_B + 1] + L[S_B + 2] * L[S_B + 2]);
        eintr = eintr - 0.5 * (R[S_B] * R[S_B] + R[S_B + 1] * R[S_B + 1] + R[S_B + 2] * R[S_B + 2]);
      }
      const double em = sm.P[Q_EINT][rm], e0 = sm.P[Q_EINT][r], ep = sm.P[Q_EINT][rp];
      if (eintl >= fmax2(em, e0) || eintl <= fmin2(em, e0) || eintr >= fmax2(e0, ep) || eintr <= fmin2(e0, ep)) {
#pragma unroll
        for (int q = 0; q < NS; q++) sl[q] = 0.0;
      }
    }
#pragma unroll
    for (int q = 0; q < nsl; q++) sm.S[q][w] = (float)sl[q];
  }
  __syncthreads();

  for (int w = tid; w < NFB; w += TL::NT) {
    const int fx = w % FBX, fy = (w / FBX) % FBY, fz = w / (FBX * FBY);
    int fc[3] = {fx, fy, fz};
    const int f = fc[AX];
    if (f > T[AX] || fx >= T[0] + (AX == 0) || fy >= T[1] + (AX == 1) || fz >= T[2] + (AX == 2)) continue;
    int lL[3] = {fx, fy, fz};
    lL[AX] = f - 1;
    int lR[3] = {lL[0], lL[1], lL[2]};
    lR[AX] = f;
    const int rL = TL::pidx(lL[0], lL[1], lL[2]), rR = TL::pidx(lR[0], lR[1], lR[2]);
    const int sL = fx + SBX * (fy + SBY * fz);
    const int sR = sL + SSTR;
    const int gL = t0[AX] + f - 1;
    const double dx1 = g.hr[gL + 2], dx2 = g.hl[gL + 3];
    // face states in FP64 (cell values + FP32 slopes)
    const double dl = sm.P[Q_D][rL] + dx1 * (double)sm.S[S_D][sL];
    const double dr = sm.P[Q_D][rR] - dx2 * (double)sm.S[S_D][sR];
    const double el = sm.P[Q_E][rL] + dx1 * (double)sm.S[S_E][sL];
    const double er = sm.P[Q_E][rR] - dx2 * (double)sm.S[S_E][sR];
    const double rdl = rcp_nr(dl), rdr = rcp_nr(dr);
    const double v1l = (sm.P[Q_M + cn][rL] + dx1 * (double)sm.S[S_M + cn][sL]) * rdl;
    const double v1r = (sm.P[Q_M + cn][rR] - dx2 * (double)sm.S[S_M + cn][sR]) * rdr;
    const double v2l = (sm.P[Q_M + c1][rL] + dx1 * (double)sm.S[S_M + c1][sL]) * rdl;
    const double v2r = (sm.P[Q_M + c1][rR] - dx2 * (double)sm.S[S_M + c1][sR]) * rdr;
    const double v3l = (sm.P[Q_M + c2][rL] + dx1 * (double)sm.S[S_M + c2][sL]) * rdl;
    const double v3r = (sm.P[Q_M + c2][rR] - dx2 * (double)sm.S[S_M + c2][sR]) * rdr;
    double b1l = 0.0, b1r = 0.0, b2l = 0.0, b2r = 0.0, b3l = 0.0, b3r = 0.0, phil = 0.0, phir = 0.0;
    if (MAG) {
      b1l = sm.P[Q_B + cn][rL] + dx1 * (double)sm.S[S_B + cn][sL];
      b1r = sm.P[Q_B + cn][rR] - dx2 * (double)sm.S[S_B + cn][sR];
      b2l = sm.P[Q_B + c1][rL] + dx1 * (double)sm.S[S_B + c1][sL];
      b2r = sm.P[Q_B + c1][rR] - dx2 * (double)sm.S[S_B + c1][sR];
      b3l = sm.P[Q_B + c2][rL] + dx1 * (double)sm.S[S_B + c2][sL];
      b3r = sm.P[Q_B + c2][rR] - dx2 * (double)sm.S[S_B + c2][sR];
      phil = sm.P[Q_PHI][rL];
      phir = sm.P[Q_PHI][rR];
    }
    // pressure recovery in FP64
    const double eil = get_eint<MAG>(el, dl, v1l, v2l, v3l, b1l, b2l, b3l);
    const double eir = get_eint<MAG>(er, dr, v1r, v2r, v3r, b1r, b2r, b3r);
    float fl[9];
    if (eil <= 0.0 || dl <= 0.0 || eir <= 0.0 || dr <= 0.0) {
      int gi[3] = {t0[0] + fx, t0[1] + fy, t0[2] + fz};
      gi[AX] = gL;
      if (atomicCAS(&A.sc->err_code, 0, kENEG_EINT) == 0) {
        A.sc->err_i = gi[0];
        A.sc->err_j = gi[1];
        A.sc->err_k = gi[2];
      }
#pragma unroll
      for (int q = 0; q < 9; q++) fl[q] = 0.0f;
    } else {
      // EOS, fast speeds and HLLD in FP32
      const float gam = (float)A.gamma;
      const float dlf = (float)dl, drf = (float)dr;
      const float ptl0 = (float)(A.gm1 * eil), ptr0 = (float)(A.gm1 * eir);
      const float b1lf = (float)b1l, b1rf = (float)b1r, b2lf = (float)b2l, b2rf = (float)b2r;
      const float b3lf = (float)b3l, b3rf = (float)b3r;
      const float csl = sqrtf(gam * ptl0 / dlf), csr = sqrtf(gam * ptr0 / drf);
      const float ptl = ptl0 + 0.5f * (b1lf * b1lf + b2lf * b2lf + b3lf * b3lf);
      const float ptr = ptr0 + 0.5f * (b1rf * b1rf + b2rf * b2rf + b3rf * b3rf);
      const float cfl = get_cf(dlf, csl, b1lf, b2lf, b3lf);
      const float cfr = get_cf(drf, csr, b1rf, b2rf, b3rf);
      hlld<float>(fl, cfl, cfr, (float)v1l, (float)v1r, (float)v2l, (float)v2r, (float)v3l, (float)v3r, dlf, drf,
                  (float)el, (float)er, ptl, ptr, b1lf, b1rf, b2lf, b2rf, b3lf, b3rf, (float)phil, (float)phir, ch);
    }
    if (AX == 2 && G.fb != nullptr && t0[2] + f == 0) {  // boundary code 10 (fluxboundary.f90:42-87)
#pragma unroll
      for (int q = 0; q < 9; q++) sm.F[q][w] = (float)G.fb[q];
      continue;
    }
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
  }
  __syncthreads();

  if (tid < TL::NC) {
    const int cx = tid % TX, cy = (tid / TX) % TY, cz = tid / (TX * TY);
    const int cc[3] = {cx, cy, cz};
    if (cx < T[0] && cy < T[1] && cz < T[2]) {
      const int wm = cx + FBX * (cy + FBY * cz);
      const int wp = wm + FSTR;
      constexpr int nv = MAG ? (GLM ? 9 : 8) : 5;
      if constexpr (SPH) {  // FP64 metric weights on the FP32 fluxes
        double cw, fm, fp;
        sph_div_weights<AX>(G, cx + t0[0], cy + t0[1], cz + t0[2], cw, fm, fp);
#pragma unroll
        for (int q = 0; q < nv; q++)
          acc[q] = acc[q] + cw * (fm * (double)sm.F[q][wm] - fp * (double)sm.F[q][wp]);
      } else {
        const double idxi = g.idxi[cc[AX] + t0[AX] + 2];
#pragma unroll
        for (int q = 0; q < nv; q++) acc[q] = acc[q] + idxi * ((double)sm.F[q][wm] - (double)sm.F[q][wp]);
      }
    }
  }
  // No barrier: the next axis's slope phase writes only S, whose last
  // reader (this axis's face phase) finished before the barrier above, and
  // its own barrier orders these reads of F before F is rewritten.  Dropping
  // it makes the mixed stage 2 % faster.
}

// One tile of one RK stage; `tile_id` enumerates the tiles of the grid
// (x fastest).  Shared by the single-grid and the batched kernels.
template <bool MAG, bool GLM, class TL, bool SPH = false, bool PUSH = false>
__device__ __forceinline__ void stage_tile_mixed(const GridDev& G, const StageArgs& A, SmemMixed<TL>& sm, int tile_id,
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
  {  // ask L2 for the U this thread's epilogue reads, while the axis passes run
    const int tid0 = threadIdx.x;
    if (tid0 < TL::NC) {
      const int cx = tid0 % TL::TX, cy = (tid0 / TL::TX) % TL::TY, cz = tid0 / (TL::TX * TL::TY);
      if (cx < T[0] && cy < T[1] && cz < T[2]) {
        const size_t c = cidx(G, t0[0] + cx, t0[1] + cy, t0[2] + cz);
        constexpr int nvp = MAG ? (GLM ? 9 : 8) : 5;
#pragma unroll
        for (int q = 0; q < nvp; q++) {
          asm volatile("prefetch.L2 [%0];" ::"l"(A.uorg + q * A.plane + c));
          if (A.ucur != A.uorg) asm volatile("prefetch.L2 [%0];" ::"l"(A.ucur + q * A.plane + c));
        }
      }
    }
  }
  stage_region<MAG, GLM, TL>(G, A, sm.P, &sm.bar, tm, t0, T);
  double acc[9];
#pragma unroll
  for (int q = 0; q < 9; q++) acc[q] = 0.0;
  const float ch = (float)A.sc->ch;
  if (TL::TX > 1 && G.solve[0]) axis_pass_mixed<0, MAG, GLM, TL, SPH>(G, A, sm, t0, T, acc, ch);
  if (TL::TY > 1 && G.solve[1]) axis_pass_mixed<1, MAG, GLM, TL, SPH>(G, A, sm, t0, T, acc, ch);
  if (TL::TZ > 1 && G.solve[2]) axis_pass_mixed<2, MAG, GLM, TL, SPH>(G, A, sm, t0, T, acc, ch);

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
      // gravity source in FP64 (source.f90:70-85 with get_fieldforce :177-228)
      const double d = A.pin[c];
      const double v[3] = {A.pin[PV * pl + c], A.pin[(PV + 1) * pl + c], A.pin[(PV + 2) * pl + c]};
      double frc[3];
      const int ijk[3] = {i, j, k};
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const AxisGeo& g = G.g[a];
        const int s = ijk[a];
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
            ph[o + 1] = A.gphi[c] * sqrt(xe * xe + ye * ye + ze * ze) / sqrt(xg * xg + yg * yg + zg * zg);
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
    const double a = __dmul_rn(A.faco, A.uorg[q * pl + c]);
    const double b = __dmul_rn(A.facn, A.ucur[q * pl + c]);
    const double t = __dmul_rn(dtf, acc[q]);
    double s1, e1, s2, e2;
    two_sum(a, b, s1, e1);
    two_sum(s1, t, s2, e2);
    const double val = __dadd_rn(s2, __dadd_rn(e1, e2));
    un[q] = val;
    A.uout[q * pl + c] = val;
  }
  const double d = un[0];
  const double rd = rcp_nr(d);
  const double v1 = un[1] * rd, v2 = un[2] * rd, v3 = un[3] * rd;
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
  if (eint <= 0.0 && atomicCAS(&A.sc->err_code, 0, kENEG_EINT) == 0) {
    A.sc->err_i = i;
    A.sc->err_j = j;
    A.sc->err_k = k;
  }
  if constexpr (PUSH) push_boundary_layers(G, A, Po, c, i, j, k);
}

template <bool MAG, bool GLM, class TL, bool SPH = false, bool PUSH = false>
__global__ void __launch_bounds__(TL::NT, TL::MINB) stage_kernel_mixed(const GridDev G, const StageArgs A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SmemMixed<TL>& sm = *reinterpret_cast<SmemMixed<TL>*>(smem_raw);
  if (A.sc->done) return;
  stage_tile_mixed<MAG, GLM, TL, SPH, PUSH>(G, A, sm, blockIdx.x, nullptr);
}

// the same stage with the stencil region staged by TMA (3-D tiles)
template <bool MAG, bool GLM, class TL>
__global__ void __launch_bounds__(TL::NT, TL::MINB)
    stage_kernel_mixed_tma(const GridDev G, const StageArgs A, const __grid_constant__ TmaMaps tm) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SmemMixed<TL>& sm = *reinterpret_cast<SmemMixed<TL>*>(smem_raw);
  if (A.sc->done) return;
  const bool tma = (smem_addr(&sm.P[0][0]) & 127u) == 0;
  stage_tile_mixed<MAG, GLM, TL>(G, A, sm, blockIdx.x, tma ? &tm : nullptr);
}

template <bool MAG, bool GLM, class TL>
static cudaError_t launch_mixed_t(const GridDev& G, const StageArgs& A, const TmaMaps* tm, cudaStream_t st) {
  constexpr int smem = (int)sizeof(SmemMixed<TL>);
  const int blocks = A.tiles[0] * A.tiles[1] * A.tiles[2];
  if constexpr (TL::HX && TL::HY && TL::HZ) {  // TMA staging needs halos on all three axes
    if (tm != nullptr) {
      static bool attr_tma = false;
      if (!attr_tma) {
        cudaError_t e = cudaFuncSetAttribute(stage_kernel_mixed_tma<MAG, GLM, TL>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr_tma = true;
      }
      stage_kernel_mixed_tma<MAG, GLM, TL><<<blocks, TL::NT, smem, st>>>(G, A, *tm);
      return cudaGetLastError();
    }
  }
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel_mixed<MAG, GLM, TL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  stage_kernel_mixed<MAG, GLM, TL><<<blocks, TL::NT, smem, st>>>(G, A);
  return cudaGetLastError();
}

template <class TL>
static cudaError_t launch_mixed_tl(const GridDev& G, const StageArgs& A, bool mag, bool glm, const TmaMaps* tm,
                                   cudaStream_t st) {
  if (mag && glm) return launch_mixed_t<true, true, TL>(G, A, tm, st);
  if (mag) return launch_mixed_t<true, false, TL>(G, A, tm, st);
  return launch_mixed_t<false, false, TL>(G, A, tm, st);
}

// spherical grids: the plain (non-TMA) mixed kernel with the metric factors
template <bool MAG, bool GLM, class TL>
static cudaError_t launch_mixed_sph(const GridDev& G, const StageArgs& A, cudaStream_t st) {
  constexpr int smem = (int)sizeof(SmemMixed<TL>);
  const int blocks = A.tiles[0] * A.tiles[1] * A.tiles[2];
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel_mixed<MAG, GLM, TL, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  stage_kernel_mixed<MAG, GLM, TL, true><<<blocks, TL::NT, smem, st>>>(G, A);
  return cudaGetLastError();
}

// r always solved; 1-D grids carry no GLM wave, 2-D and 3-D MHD grids do
template <class TL>
static cudaError_t launch_mixed_sph_tl(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st) {
  constexpr bool multi = (TL::TY > 1) || (TL::TZ > 1);
  if (mag && glm != multi) return cudaErrorInvalidValue;
  if (!mag) return launch_mixed_sph<false, false, TL>(G, A, st);
  return launch_mixed_sph<true, multi, TL>(G, A, st);
}

static cudaError_t launch_mixed_spherical(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st) {
  const int* t = A.tile;
  if (t[0] == 8 && t[1] == 8 && t[2] == 8) return launch_mixed_sph_tl<Tile<8, 8, 8, 640, 1>>(G, A, mag, glm, st);
  if (t[0] == 8 && t[1] == 8 && t[2] == 4) return launch_mixed_sph_tl<Tile<8, 8, 4, 384, 2>>(G, A, mag, glm, st);
  if (t[0] == 16 && t[1] == 16 && t[2] == 1) return launch_mixed_sph_tl<Tile<16, 16, 1, 288, 2>>(G, A, mag, glm, st);
  if (t[0] == 16 && t[1] == 1 && t[2] == 16) return launch_mixed_sph_tl<Tile<16, 1, 16, 288, 2>>(G, A, mag, glm, st);
  if (t[0] == 256 && t[1] == 1 && t[2] == 1) return launch_mixed_sph_tl<Tile<256, 1, 1, 288, 2>>(G, A, mag, glm, st);
  return cudaErrorInvalidValue;
}

// z slabs exchanging by push (see push_boundary_layers): 3-D Cartesian tiles
template <bool MAG, bool GLM, class TL>
static cudaError_t launch_mixed_push_t(const GridDev& G, const StageArgs& A, cudaStream_t st) {
  constexpr int smem = (int)sizeof(SmemMixed<TL>);
  const int blocks = A.tiles[0] * A.tiles[1] * A.tiles[2];
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel_mixed<MAG, GLM, TL, false, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  stage_kernel_mixed<MAG, GLM, TL, false, true><<<blocks, TL::NT, smem, st>>>(G, A);
  return cudaGetLastError();
}

static cudaError_t launch_mixed_push(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st) {
  const int* t = A.tile;
  if (G.sph.on || t[2] == 1) return cudaErrorInvalidValue;
  using T4 = Tile<8, 8, 4, 384, 2>;
  using T8 = Tile<8, 8, 8, 640, 1>;
  const bool t884 = t[0] == 8 && t[1] == 8 && t[2] == 4, t888 = t[0] == 8 && t[1] == 8 && t[2] == 8;
  if (!t884 && !t888) return cudaErrorInvalidValue;
  if (mag && glm) return t884 ? launch_mixed_push_t<true, true, T4>(G, A, st) : launch_mixed_push_t<true, true, T8>(G, A, st);
  if (mag) return t884 ? launch_mixed_push_t<true, false, T4>(G, A, st) : launch_mixed_push_t<true, false, T8>(G, A, st);
  return t884 ? launch_mixed_push_t<false, false, T4>(G, A, st) : launch_mixed_push_t<false, false, T8>(G, A, st);
}

cudaError_t launch_stage_mixed(const GridDev& G, const StageArgs& A, bool mag, bool glm, const TmaMaps* tm,
                               cudaStream_t st) {
  if (A.push[0] != nullptr || A.push[1] != nullptr) return launch_mixed_push(G, A, mag, glm, st);
  if (G.sph.on) return launch_mixed_spherical(G, A, mag, glm, st);
  const int* t = A.tile;
  if (t[0] == 8 && t[1] == 8 && t[2] == 8) return launch_mixed_tl<Tile<8, 8, 8, 640, 1>>(G, A, mag, glm, tm, st);
  if (t[0] == 8 && t[1] == 8 && t[2] == 4) return launch_mixed_tl<Tile<8, 8, 4, 384, 2>>(G, A, mag, glm, tm, st);
  if (t[0] == 16 && t[1] == 16 && t[2] == 1) return launch_mixed_tl<Tile<16, 16, 1, 288, 3>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 16 && t[1] == 1 && t[2] == 16) return launch_mixed_tl<Tile<16, 1, 16, 288, 3>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 16 && t[2] == 16) return launch_mixed_tl<Tile<1, 16, 16, 288, 3>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 256 && t[1] == 1 && t[2] == 1) return launch_mixed_tl<Tile<256, 1, 1, 288, 3>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 256 && t[2] == 1) return launch_mixed_tl<Tile<1, 256, 1, 288, 3>>(G, A, mag, glm, nullptr, st);
  if (t[0] == 1 && t[1] == 1 && t[2] == 256) return launch_mixed_tl<Tile<1, 1, 256, 288, 3>>(G, A, mag, glm, nullptr, st);
  return cudaErrorInvalidValue;
}

// batched form (see batch_stage_kernel in hmn_kernels.cu)
template <bool MAG, bool GLM, class TL, bool DYN>
__global__ void __launch_bounds__(TL::NT, TL::MINB) batch_stage_kernel_mixed(SimDesc* sims, const int2* items,
                                                                              int nitems, int stage, int rk,
                                                                              int* queue) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SmemMixed<TL>& sm = *reinterpret_cast<SmemMixed<TL>*>(smem_raw);
  for_each_item<DYN>(nitems, queue, [&](int it) {
    const int2 w = items[it];
    SimDesc& S = sims[w.x];
    if (!S.active || S.sc.done) return;
    const StageArgs A = batch_stage_args(S, stage, rk);
    stage_tile_mixed<MAG, GLM, TL>(S.G, A, sm, w.y, nullptr);
    __syncthreads();
  });
}

using M3D = Tile<8, 8, 8, 640, 1>;
using M3D4 = Tile<8, 8, 4, 384, 2>;
using M2D = Tile<16, 16, 1, 288, 3>;
using M2D8 = Tile<32, 8, 1, 320, 3>;
using M1D = Tile<256, 1, 1, 288, 3>;

template <bool MAG, bool GLM, class TL>
static cudaError_t bm_attr_t() {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(batch_stage_kernel_mixed<MAG, GLM, TL, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SmemMixed<TL>));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(batch_stage_kernel_mixed<MAG, GLM, TL, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SmemMixed<TL>));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  return cudaSuccess;
}

template <bool MAG, bool GLM, class TL>
static cudaError_t launch_bm_t(SimDesc* sims, const int2* items, int nitems, int stage, int rk, int grid,
                               int* queue, cudaStream_t st) {
  cudaError_t e = bm_attr_t<MAG, GLM, TL>();
  if (e != cudaSuccess) return e;
  if (queue)
    batch_stage_kernel_mixed<MAG, GLM, TL, true>
        <<<grid, TL::NT, sizeof(SmemMixed<TL>), st>>>(sims, items, nitems, stage, rk, queue);
  else
    batch_stage_kernel_mixed<MAG, GLM, TL, false>
        <<<grid, TL::NT, sizeof(SmemMixed<TL>), st>>>(sims, items, nitems, stage, rk, nullptr);
  return cudaGetLastError();
}

template <class TL>
static cudaError_t launch_bm_tl(SimDesc* sims, const int2* items, int nitems, bool mag, bool glm, int stage, int rk,
                                int grid, int* queue, cudaStream_t st) {
  if (mag && glm) return launch_bm_t<true, true, TL>(sims, items, nitems, stage, rk, grid, queue, st);
  if (mag) return launch_bm_t<true, false, TL>(sims, items, nitems, stage, rk, grid, queue, st);
  return launch_bm_t<false, false, TL>(sims, items, nitems, stage, rk, grid, queue, st);
}

cudaError_t launch_batch_stage_mixed(SimDesc* sims, const int2* items, int nitems, int tid, bool mag, bool glm,
                                     int stage, int rk, int grid, int* queue, cudaStream_t st) {
  switch (tid) {
    case 0: return launch_bm_tl<M3D>(sims, items, nitems, mag, glm, stage, rk, grid, queue, st);
    case 1: return launch_bm_tl<M3D4>(sims, items, nitems, mag, glm, stage, rk, grid, queue, st);
    case 2: return launch_bm_tl<M2D>(sims, items, nitems, mag, glm, stage, rk, grid, queue, st);
    case 3: return launch_bm_tl<M2D8>(sims, items, nitems, mag, glm, stage, rk, grid, queue, st);
    case 4: return launch_bm_tl<M1D>(sims, items, nitems, mag, glm, stage, rk, grid, queue, st);
  }
  return cudaErrorInvalidValue;
}

template <bool MAG, bool GLM, class TL>
static int occ_m() {
  int n = 0;
  bm_attr_t<MAG, GLM, TL>();
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_stage_kernel_mixed<MAG, GLM, TL, true>, TL::NT,
                                                sizeof(SmemMixed<TL>));  // the static split's is no larger
  return n > 0 ? n : 1;
}

template <class TL>
static int occ_m_tl(bool mag, bool glm) {
  if (mag && glm) return occ_m<true, true, TL>();
  if (mag) return occ_m<true, false, TL>();
  return occ_m<false, false, TL>();
}

int batch_stage_mixed_blocks_per_sm(int tid, bool mag, bool glm) {
  switch (tid) {
    case 0: return occ_m_tl<M3D>(mag, glm);
    case 1: return occ_m_tl<M3D4>(mag, glm);
    case 2: return occ_m_tl<M2D>(mag, glm);
    case 3: return occ_m_tl<M2D8>(mag, glm);
  }
  return occ_m_tl<M1D>(mag, glm);
}

}  // namespace hmn
