// hmn_kernels.cu -- FP64 kernels of the explicit MHD step for sm_100a.
//
// Compiled with --fmad=false: every operation is a single IEEE binary64
// operation in the reference's order, so results are bit-identical to the
// Fortran path (and to the CPU oracle that restates it).
//
// One RK stage (src/main/hydro.f90:35-41: boundarycondition -> numflux ->
// source -> rungekutta) is ONE launch of stage_kernel.  A CTA owns a tile of
// cells; for every solved axis it
//   1. stages the primitives of the tile plus two cells either side along
//      the axis into shared memory, generating ghost cells from the boundary
//      codes on the fly (boundarycondition.f90, codes 0-3),
//   2. computes the limited slopes of those cells (interpolation.f90),
//   3. computes the HLLD face fluxes (numflux.f90 + hlldflux.f90),
//   4. accumulates the flux divergence of its cells in shared memory,
// and finally applies the RK combination (rungekutta.f90:35-59) with the
// gravity source (source.f90:70-85) and writes the new conserved state.
// Fluxes and slopes never leave the SM.
#include <cuda_runtime.h>

#include <cstdint>

#include "hmn_internal.h"
#include "hmn_math.cuh"

namespace hmn {

// conserved slots (checksetup.f90:61-75)
enum { ICNT = 0, IMO1 = 1, IENE = 4, IMG1 = 5, I9WV = 8 };
// staged primitive quantities per cell: d, m1..3 (= d*v), e, b1..3, phi, eint
enum { Q_D = 0, Q_M = 1, Q_E = 4, Q_B = 5, Q_PHI = 8, Q_EINT = 9, NQ = 10 };
// slopes: d, e, m1..3, b1..3
enum { S_D = 0, S_E = 1, S_M = 2, S_B = 5, NS = 8 };

constexpr int kThreads = 256;
constexpr int kMaxCells = 256;   // interior cells of a tile
constexpr int kMaxRegion = 512;  // tile + 2 cells either side along one axis
constexpr int kMaxSlope = 384;   // tile + 1 cell either side
constexpr int kMaxFace = 320;    // tile + 1 face

__device__ __forceinline__ void record_error(DevScalars* sc, int code, int i, int j, int k) {
  if (atomicCAS(&sc->err_code, 0, code) == 0) {
    sc->err_i = i;
    sc->err_j = j;
    sc->err_k = k;
  }
}

__device__ __forceinline__ size_t cidx(const GridDev& G, int i, int j, int k) {
  return (size_t)i + (size_t)G.n[0] * ((size_t)j + (size_t)G.n[1] * (size_t)k);
}

// Primitives of an interior cell, derived from the state exactly as
// rungekutta.f90:205-229 (primitive) and eos.f90:805-842 (internalenergy).
template <bool MAG, bool GLM>
__device__ __forceinline__ void interior_prim(const double* src, int src_prim, size_t plane, size_t c,
                                              double phifac, double& d, double v[3], double& e, double b[3],
                                              double& phi, double& eint) {
  d = src[c];
  if (src_prim) {
    v[0] = src[plane + c];
    v[1] = src[2 * plane + c];
    v[2] = src[3 * plane + c];
  } else {
    v[0] = src[plane + c] / d;
    v[1] = src[2 * plane + c] / d;
    v[2] = src[3 * plane + c] / d;
  }
  e = src[4 * plane + c];
  if (MAG) {
    b[0] = src[5 * plane + c];
    b[1] = src[6 * plane + c];
    b[2] = src[7 * plane + c];
  } else {
    b[0] = b[1] = b[2] = 0.0;
  }
  phi = GLM ? src[8 * plane + c] * phifac : 0.0;
  eint = get_eint<MAG>(e, d, v[0], v[1], v[2], b[0], b[1], b[2]);
}

// Staged quantities of any cell of a tile's region: interior cells directly,
// ghost cells (at most one axis out of range) through the boundary codes
// (boundarycondition.f90, codes 0 periodic, 1 reflective, 2 outgoing,
// 3 free) followed by the ghost energy of boundarycondition.f90:222-243.
template <bool MAG, bool GLM>
__device__ __forceinline__ void stage_cell(const GridDev& G, const StageArgs& A, int i, int j, int k,
                                           double q[NQ]) {
  int c3[3] = {i, j, k};
  int ax = -1;
#pragma unroll
  for (int a = 0; a < 3; a++)
    if (c3[a] < 0 || c3[a] >= G.n[a]) ax = a;
  double d, v[3], e, b[3], phi, eint;
  if (ax < 0) {
    interior_prim<MAG, GLM>(A.src, A.src_prim, A.plane, cidx(G, i, j, k), A.phifac, d, v, e, b, phi, eint);
    q[Q_D] = d;
    q[Q_M + 0] = d * v[0];
    q[Q_M + 1] = d * v[1];
    q[Q_M + 2] = d * v[2];
    q[Q_E] = e;
    q[Q_B + 0] = b[0];
    q[Q_B + 1] = b[1];
    q[Q_B + 2] = b[2];
    q[Q_PHI] = phi;
    q[Q_EINT] = eint;
    return;
  }
  const int n = G.n[ax];
  const int s = c3[ax];
  const int io = s < 0 ? 0 : 1;
  const int gl = io == 0 ? s + 2 : s - n;  // ghost layer 0 or 1
  const int per = io == 0 ? n - 2 + gl : gl;
  const int refl = io == 0 ? 1 - gl : n - 1 - gl;
  const int edge = io == 0 ? 0 : n - 1;
  const int bs = G.bc[ax][io][0], bv = G.bc[ax][io][1];
  const int ss = bs == 0 ? per : (bs == 1 ? refl : edge);
  const int sv = bv == 0 ? per : (bv == 1 ? refl : edge);
  // scalar quantities (d, p, phi) from the scalar image cell
  c3[ax] = ss;
  interior_prim<MAG, GLM>(A.src, A.src_prim, A.plane, cidx(G, c3[0], c3[1], c3[2]), A.phifac, d, v, e, b, phi,
                          eint);
  const double dg = d;
  const double pg = A.gm1 * eint;  // eos.f90:256 (pressure of the image cell)
  const double phig = phi;
  // vector quantities (v, B) from the vector image cell
  if (sv != ss) {
    c3[ax] = sv;
    interior_prim<MAG, GLM>(A.src, A.src_prim, A.plane, cidx(G, c3[0], c3[1], c3[2]), A.phifac, d, v, e, b, phi,
                            eint);
  }
  double vn = v[ax];
  if (bv == 1) {
    vn = -vn;
    b[ax] = -b[ax];
  } else if (bv == 2) {
    if (io == 0) {
      vn = ax == 0 ? fmin2(0.0, vn) : vn * (0.5 - fsign(0.5, vn));  // :165 and the y/z plug form
    } else {
      vn = vn * (0.5 + fsign(0.5, vn));
    }
  }
  v[ax] = vn;
  const double eg = pg / A.gm1;  // eos.f90:287-289
  const double b1 = b[0], b2 = b[1], b3 = b[2];
  q[Q_D] = dg;
  q[Q_M + 0] = dg * v[0];
  q[Q_M + 1] = dg * v[1];
  q[Q_M + 2] = dg * v[2];
  q[Q_E] = eg + 0.5 * (dg * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + b1 * b1 + b2 * b2 + b3 * b3);
  q[Q_B + 0] = b1;
  q[Q_B + 1] = b2;
  q[Q_B + 2] = b3;
  q[Q_PHI] = phig;
  q[Q_EINT] = eg;
}

struct Smem {
  double P[NQ][kMaxRegion];
  double S[NS][kMaxSlope];
  double F[9][kMaxFace];
  double acc[9][kMaxCells];
};

template <bool MAG, bool GLM>
__global__ void __launch_bounds__(kThreads, 2) stage_kernel(const GridDev G, const StageArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x;
  if (A.sc->done) return;

  // tile origin and effective extent
  int bid = blockIdx.x;
  int t0[3], T[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    int ti = bid % A.tiles[a];
    bid /= A.tiles[a];
    t0[a] = ti * A.tile[a];
    T[a] = min(A.tile[a], G.n[a] - t0[a]);
  }
  const int ncell = T[0] * T[1] * T[2];
  const int nvar = A.nvar;
  for (int w = tid; w < ncell; w += kThreads)
    for (int q = 0; q < 9; q++) sm.acc[q][w] = 0.0;

  const double ch = A.sc->ch;
  const int nsl = MAG ? NS : S_B;

  for (int a = 0; a < 3; a++) {
    if (!G.solve[a]) continue;
    const AxisGeo& g = G.g[a];
    // ---- 1. stage the region (tile +-2 along a) ---------------------------
    int R[3] = {T[0], T[1], T[2]};
    R[a] += 4;
    int r0[3] = {t0[0], t0[1], t0[2]};
    r0[a] -= 2;
    const int nreg = R[0] * R[1] * R[2];
    __syncthreads();  // previous axis finished with P/S/F
    for (int w = tid; w < nreg; w += kThreads) {
      int rx = w % R[0], ry = (w / R[0]) % R[1], rz = w / (R[0] * R[1]);
      double q[NQ];
      stage_cell<MAG, GLM>(G, A, r0[0] + rx, r0[1] + ry, r0[2] + rz, q);
#pragma unroll
      for (int k = 0; k < NQ; k++) sm.P[k][w] = q[k];
    }
    const int rstride = a == 0 ? 1 : (a == 1 ? R[0] : R[0] * R[1]);
    __syncthreads();

    // ---- 2. limited slopes for the tile +-1 along a -----------------------
    int SB[3] = {T[0], T[1], T[2]};
    SB[a] += 2;
    const int nsb = SB[0] * SB[1] * SB[2];
    const int sstride = a == 0 ? 1 : (a == 1 ? SB[0] : SB[0] * SB[1]);
    for (int w = tid; w < nsb; w += kThreads) {
      int sx = w % SB[0], sy = (w / SB[0]) % SB[1], sz = w / (SB[0] * SB[1]);
      int rc[3] = {sx, sy, sz};
      rc[a] += 1;
      const int r = rc[0] + R[0] * (rc[1] + R[1] * rc[2]);
      const int cg = (a == 0 ? sx : (a == 1 ? sy : sz)) + t0[a] - 1;  // global coordinate along a
      double sl[NS];
      if (A.limiter == 0) {
#pragma unroll
        for (int k = 0; k < NS; k++) sl[k] = 0.0;
      } else {
        const double hl = g.hl[cg + 2], hr = g.hr[cg + 2];
        double L[NS], Rv[NS];
        // slope inputs in the order d, e, m1, m2, m3, b1, b2, b3
        const int qmap[NS] = {Q_D, Q_E, Q_M + 0, Q_M + 1, Q_M + 2, Q_B + 0, Q_B + 1, Q_B + 2};
        if (A.limiter == 1) {
          const double i0 = g.idx[cg + 2], i1 = g.idx[cg + 3], is = g.isum[cg + 2];
#pragma unroll
          for (int k = 0; k < NS; k++) {
            if (k >= nsl) { sl[k] = 0.0; continue; }
            const double u0 = sm.P[qmap[k]][r - rstride], u1 = sm.P[qmap[k]][r], u2 = sm.P[qmap[k]][r + rstride];
            const double du = lim_minmod(u0, u1, u2, i0, i1, is);
            sl[k] = du;
            L[k] = u1 - hl * du;
            Rv[k] = u1 + hr * du;
          }
        } else {
          const double cf = g.mcf[cg + 2], cb = g.mcb[cg + 2], ga = g.ga[cg + 2], gb = g.gb[cg + 2];
#pragma unroll
          for (int k = 0; k < NS; k++) {
            if (k >= nsl) { sl[k] = 0.0; continue; }
            const double u0 = sm.P[qmap[k]][r - rstride], u1 = sm.P[qmap[k]][r], u2 = sm.P[qmap[k]][r + rstride];
            const double du = lim_mmc(u0, u1, u2, cf, cb, ga, gb);
            sl[k] = du;
            L[k] = u1 - hl * du;
            Rv[k] = u1 + hr * du;
          }
        }
        // admissibility of the face internal energies (interpolation.f90:147-163)
        double eintl = L[S_E] - 0.5 * (L[S_M] * L[S_M] + L[S_M + 1] * L[S_M + 1] + L[S_M + 2] * L[S_M + 2]) / L[S_D];
        double eintr =
            Rv[S_E] - 0.5 * (Rv[S_M] * Rv[S_M] + Rv[S_M + 1] * Rv[S_M + 1] + Rv[S_M + 2] * Rv[S_M + 2]) / Rv[S_D];
        if (MAG) {
          eintl = eintl - 0.5 * (L[S_B] * L[S_B] + L[S_B + 1] * L[S_B + 1] + L[S_B + 2] * L[S_B + 2]);
          eintr = eintr - 0.5 * (Rv[S_B] * Rv[S_B] + Rv[S_B + 1] * Rv[S_B + 1] + Rv[S_B + 2] * Rv[S_B + 2]);
        }
        const double em = sm.P[Q_EINT][r - rstride], e0 = sm.P[Q_EINT][r], ep = sm.P[Q_EINT][r + rstride];
        if (eintl >= fmax2(em, e0) || eintl <= fmin2(em, e0) || eintr >= fmax2(e0, ep) || eintr <= fmin2(e0, ep)) {
#pragma unroll
          for (int k = 0; k < NS; k++) sl[k] = 0.0;
        }
      }
#pragma unroll
      for (int k = 0; k < NS; k++) sm.S[k][w] = sl[k];
    }
    __syncthreads();

    // ---- 3. HLLD fluxes on the T+1 faces along a ---------------------------
    int FB[3] = {T[0], T[1], T[2]};
    FB[a] += 1;
    const int nfb = FB[0] * FB[1] * FB[2];
    const int cn = a, c1 = (a + 1) % 3, c2 = (a + 2) % 3;  // normal and tangential components
    for (int w = tid; w < nfb; w += kThreads) {
      int fx = w % FB[0], fy = (w / FB[0]) % FB[1], fz = w / (FB[0] * FB[1]);
      int fc[3] = {fx, fy, fz};
      const int f = fc[a];
      // left cell: slope-box coordinate f along a, region coordinate f+1
      int sc3[3] = {fx, fy, fz};
      const int sL = sc3[0] + SB[0] * (sc3[1] + SB[1] * sc3[2]);
      const int sR = sL + sstride;
      int rc[3] = {fx, fy, fz};
      rc[a] += 1;
      const int rL = rc[0] + R[0] * (rc[1] + R[1] * rc[2]);
      const int rR = rL + rstride;
      const int gLc = t0[a] - 1 + f;  // global coordinate of the left cell
      const double dx1 = g.hr[gLc + 2];      // xi(i)-x(i)
      const double dx2 = g.hl[gLc + 3];      // x(i+1)-xi(i)
      const double dl = sm.P[Q_D][rL] + dx1 * sm.S[S_D][sL];
      const double dr = sm.P[Q_D][rR] - dx2 * sm.S[S_D][sR];
      const double el = sm.P[Q_E][rL] + dx1 * sm.S[S_E][sL];
      const double er = sm.P[Q_E][rR] - dx2 * sm.S[S_E][sR];
      const double v1l = (sm.P[Q_M + cn][rL] + dx1 * sm.S[S_M + cn][sL]) / dl;
      const double v1r = (sm.P[Q_M + cn][rR] - dx2 * sm.S[S_M + cn][sR]) / dr;
      const double v2l = (sm.P[Q_M + c1][rL] + dx1 * sm.S[S_M + c1][sL]) / dl;
      const double v2r = (sm.P[Q_M + c1][rR] - dx2 * sm.S[S_M + c1][sR]) / dr;
      const double v3l = (sm.P[Q_M + c2][rL] + dx1 * sm.S[S_M + c2][sL]) / dl;
      const double v3r = (sm.P[Q_M + c2][rR] - dx2 * sm.S[S_M + c2][sR]) / dr;
      double b1l = 0.0, b1r = 0.0, b2l = 0.0, b2r = 0.0, b3l = 0.0, b3r = 0.0, phil = 0.0, phir = 0.0;
      if (MAG) {
        b1l = sm.P[Q_B + cn][rL] + dx1 * sm.S[S_B + cn][sL];
        b1r = sm.P[Q_B + cn][rR] - dx2 * sm.S[S_B + cn][sR];
        b2l = sm.P[Q_B + c1][rL] + dx1 * sm.S[S_B + c1][sL];
        b2r = sm.P[Q_B + c1][rR] - dx2 * sm.S[S_B + c1][sR];
        b3l = sm.P[Q_B + c2][rL] + dx1 * sm.S[S_B + c2][sL];
        b3r = sm.P[Q_B + c2][rR] - dx2 * sm.S[S_B + c2][sR];
        // phi is never reconstructed: its slope is identically zero (allocations.f90)
        phil = sm.P[Q_PHI][rL] + dx1 * 0.0;
        phir = sm.P[Q_PHI][rR] - dx2 * 0.0;
      }
      const double eil = get_eint<MAG>(el, dl, v1l, v2l, v3l, b1l, b2l, b3l);
      const double eir = get_eint<MAG>(er, dr, v1r, v2r, v3r, b1r, b2r, b3r);
      double fl[9];
      if (eil <= 0.0 || dl <= 0.0 || eir <= 0.0 || dr <= 0.0) {
        int gi[3] = {t0[0] + fx, t0[1] + fy, t0[2] + fz};
        gi[a] = gLc;
        record_error(A.sc, kENEG_EINT, gi[0], gi[1], gi[2]);  // numflux.f90:117 -> error_flux
#pragma unroll
        for (int k = 0; k < 9; k++) fl[k] = 0.0;
      } else {
        // eos_p_cs (eos.f90:209-219) with erad = 0
        const double ptl0 = A.gm1 * eil, ptr0 = A.gm1 * eir;
        const double csl = sqrt(A.gamma * ptl0 / dl), csr = sqrt(A.gamma * ptr0 / dr);
        const double ptl = ptl0 + 0.5 * (b1l * b1l + b2l * b2l + b3l * b3l);
        const double ptr = ptr0 + 0.5 * (b1r * b1r + b2r * b2r + b3r * b3r);
        const double cfl = get_cf(dl, csl, b1l, b2l, b3l);
        const double cfr = get_cf(dr, csr, b1r, b2r, b3r);
        hlld(fl, cfl, cfr, v1l, v1r, v2l, v2r, v3l, v3r, dl, dr, el, er, ptl, ptr, b1l, b1r, b2l, b2r, b3l, b3r,
             phil, phir, ch);
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
    }
    __syncthreads();

    // ---- 4. flux divergence along a ---------------------------------------
    const int fstride = a == 0 ? 1 : (a == 1 ? FB[0] : FB[0] * FB[1]);
    for (int w = tid; w < ncell; w += kThreads) {
      int cx = w % T[0], cy = (w / T[0]) % T[1], cz = w / (T[0] * T[1]);
      const int wm = cx + FB[0] * (cy + FB[1] * cz);  // face on the low side
      const int wp = wm + fstride;
      const int cga = (a == 0 ? cx : (a == 1 ? cy : cz)) + t0[a];
      const double idxi = g.idxi[cga + 2];
      for (int q = 0; q < nvar; q++) sm.acc[q][w] = sm.acc[q][w] + idxi * (sm.F[q][wm] - sm.F[q][wp]);
    }
  }
  __syncthreads();

  // ---- RK combination (rungekutta.f90:35-59) + source (source.f90:70-85) ---
  const double dtf = A.fact * A.sc->dt;
  for (int w = tid; w < ncell; w += kThreads) {
    int cx = w % T[0], cy = (w / T[0]) % T[1], cz = w / (T[0] * T[1]);
    const int i = t0[0] + cx, j = t0[1] + cy, k = t0[2] + cz;
    const size_t c = cidx(G, i, j, k);
    double src[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const bool grav = A.gphi != nullptr;
    if (grav) {
      double d, v[3], e, b[3], phi, eint;
      interior_prim<MAG, GLM>(A.src, A.src_prim, A.plane, c, A.phifac, d, v, e, b, phi, eint);
      double frc[3];
      int ijk[3] = {i, j, k};
      for (int a = 0; a < 3; a++) {
        const AxisGeo& g = G.g[a];
        const int s = ijk[a];
        // neighbours of the potential with the ghost images of the
        // boundary (periodic copy, or phi ~ 1/r elsewhere)
        double ph[3];
        for (int o = -1; o <= 1; o++) {
          int nb[3] = {i, j, k};
          nb[a] = s + o;
          if (nb[a] >= 0 && nb[a] < G.n[a]) {
            ph[o + 1] = A.gphi[cidx(G, nb[0], nb[1], nb[2])];
          } else if (G.bc[a][0][0] == 0) {
            nb[a] = nb[a] < 0 ? G.n[a] - 1 : 0;
            ph[o + 1] = A.gphi[cidx(G, nb[0], nb[1], nb[2])];
          } else {
            // Robin image phi_g = phi_edge * r_edge / r_g
            int ed[3] = {i, j, k};
            const double xe = G.g[0].x[ed[0] + 2], ye = G.g[1].x[ed[1] + 2], ze = G.g[2].x[ed[2] + 2];
            const double xg = G.g[0].x[nb[0] + 2], yg = G.g[1].x[nb[1] + 2], zg = G.g[2].x[nb[2] + 2];
            const double re = sqrt(xe * xe + ye * ye + ze * ze), rg = sqrt(xg * xg + yg * yg + zg * zg);
            ph[o + 1] = A.gphi[c] * re / rg;
          }
        }
        const double dxm = g.dx[s + 2], dxp = g.dx[s + 3], im = g.idx[s + 2], ip = g.idx[s + 3];
        frc[a] = -((dxm * ip * ph[2] - dxp * im * ph[0]) / (dxm + dxp) + (dxp - dxm) * im * ip * ph[1]) * d;
      }
      src[1] = frc[0];
      src[2] = frc[1];
      src[3] = frc[2];
      src[4] = frc[0] * v[0] + frc[1] * v[1] + frc[2] * v[2];
    }
    double un[9];
    for (int q = 0; q < nvar; q++) {
      double s = sm.acc[q][w];
      if (grav && q >= 1 && q <= 4) s = s + src[q];
      const double val = A.faco * A.uorg[q * A.plane + c] + A.facn * A.ucur[q * A.plane + c] + dtf * s;
      un[q] = val;
      A.uout[q * A.plane + c] = val;
    }
    // primitive + internalenergy check of the new state (eos.f90:833-839)
    const double d = un[0];
    const double v1 = un[1] / d, v2 = un[2] / d, v3 = un[3] / d;
    const double eint =
        get_eint<MAG>(un[4], d, v1, v2, v3, MAG ? un[5] : 0.0, MAG ? un[6] : 0.0, MAG ? un[7] : 0.0);
    if (eint <= 0.0) record_error(A.sc, kENEG_EINT, i, j, k);
  }
}

// ---------------------------------------------------------------------------
// CFL timestep (timestep.f90:45-98, dti_cell :125-183)

__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

template <bool MAG, bool GLM>
__global__ void __launch_bounds__(256) cfl_kernel(const GridDev G, const double* src, int src_prim, size_t plane,
                                                  double gamma, DevScalars* sc) {
  if (sc->done) return;
  const double gm1 = gamma - 1.0;
  const size_t ncell = plane;
  double my_dti = __longlong_as_double(0x7ff0000000000000LL);  // +inf
  double my_cf = 0.0;
  const double off0 = G.solve[0] ? 1.0 : 0.0, off1 = G.solve[1] ? 1.0 : 0.0, off2 = G.solve[2] ? 1.0 : 0.0;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % G.n[0]);
    const int j = (int)((c / G.n[0]) % G.n[1]);
    const int k = (int)(c / ((size_t)G.n[0] * G.n[1]));
    double d, v[3], e, b[3], phi, eint;
    interior_prim<MAG, GLM>(src, src_prim, plane, c, 1.0, d, v, e, b, phi, eint);
    if (eint <= 0.0 || d <= 0.0) {
      record_error(sc, kENEG_EINT, i, j, k);
      continue;
    }
    const double p = gm1 * eint;
    const double cs = sqrt(gamma * p / d);
    double cf1, cf2, cf3;
    if (MAG) {
      cf1 = get_cf(d, cs, b[0], b[1], b[2]) + fabs(v[0]);
      cf2 = get_cf(d, cs, b[1], b[0], b[2]) + fabs(v[1]);
      cf3 = get_cf(d, cs, b[2], b[0], b[1]) + fabs(v[2]);
    } else {
      cf1 = cs + fabs(v[0]);
      cf2 = cs + fabs(v[1]);
      cf3 = cs + fabs(v[2]);
    }
    const double dxi1 = G.g[0].dxi[i + 2], dxi2 = G.g[1].dxi[j + 2], dxi3 = G.g[2].dxi[k + 2];
    const double dvol = dxi1 * dxi2 * dxi3;  // metric.f90:45-48
    const double sa1 = dxi2 * dxi3, sa2 = dxi1 * dxi3, sa3 = dxi1 * dxi2;
    const double dti = dvol / (cf1 * off0 * (sa1 + sa1) + cf2 * off1 * (sa2 + sa2) + cf3 * off2 * (sa3 + sa3));
    const double cm = fmax2(fmax2(cf1, cf2), cf3);
    my_cf = fmax2(my_cf, cm);
    my_dti = fmin2(my_dti, dti);
  }
  // warp then block reduction; min/max are exact so the order is irrelevant
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
      atomicMin(&sc->min_dti_bits, dbits(my_dti));
      atomicMax(&sc->cfmax_bits, dbits(my_cf));
    }
  }
}

// dt from the reduced values, with the output/end-time clamps
// (timestep.f90:74-98).  One thread; also re-arms the reduction slots.
__global__ void cfl_finalize_kernel(DevScalars* sc) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || sc->done) return;
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

// ---------------------------------------------------------------------------
// layout kernels: primitives of the current state for download

template <bool MAG, bool GLM>
__global__ void prim_kernel(const GridDev G, const double* src, int src_prim, size_t plane, double phifac,
                            double* out /* 9 planes d,v1,v2,v3,e,b1,b2,b3,phi */, double* p_out, double gm1) {
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < plane; c += (size_t)gridDim.x * blockDim.x) {
    double d, v[3], e, b[3], phi, eint;
    interior_prim<MAG, GLM>(src, src_prim, plane, c, phifac, d, v, e, b, phi, eint);
    out[c] = d;
    out[plane + c] = v[0];
    out[2 * plane + c] = v[1];
    out[3 * plane + c] = v[2];
    out[4 * plane + c] = e;
    out[5 * plane + c] = b[0];
    out[6 * plane + c] = b[1];
    out[7 * plane + c] = b[2];
    out[8 * plane + c] = phi;
    if (p_out) p_out[c] = gm1 * eint;
  }
}

// ---------------------------------------------------------------------------
// host-side launchers (called from hmn_capi.cu)

size_t stage_smem_bytes() { return sizeof(Smem); }

// time += dt; tn += 1; end check (hormone.f90:147-155) on the device clock
__global__ void advance_kernel(DevScalars* sc) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || sc->done) return;
  sc->time = sc->time + sc->dt;
  sc->tn = sc->tn + 1;
  if (sc->endstyle == 1 && sc->time >= sc->t_end) sc->done = 1;
}

cudaError_t launch_advance(DevScalars* sc, cudaStream_t st) {
  advance_kernel<<<1, 32, 0, st>>>(sc);
  return cudaGetLastError();
}

template <bool MAG, bool GLM>
static cudaError_t launch_stage_t(const GridDev& G, const StageArgs& A, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<MAG, GLM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(Smem));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int blocks = A.tiles[0] * A.tiles[1] * A.tiles[2];
  stage_kernel<MAG, GLM><<<blocks, kThreads, sizeof(Smem), st>>>(G, A);
  return cudaGetLastError();
}

cudaError_t launch_stage(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st) {
  if (mag && glm) return launch_stage_t<true, true>(G, A, st);
  if (mag) return launch_stage_t<true, false>(G, A, st);
  return launch_stage_t<false, false>(G, A, st);
}

cudaError_t launch_cfl(const GridDev& G, const double* src, int src_prim, size_t plane, double gamma,
                       DevScalars* sc, bool mag, bool glm, int nblocks, cudaStream_t st) {
  if (mag && glm)
    cfl_kernel<true, true><<<nblocks, 256, 0, st>>>(G, src, src_prim, plane, gamma, sc);
  else if (mag)
    cfl_kernel<true, false><<<nblocks, 256, 0, st>>>(G, src, src_prim, plane, gamma, sc);
  else
    cfl_kernel<false, false><<<nblocks, 256, 0, st>>>(G, src, src_prim, plane, gamma, sc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  cfl_finalize_kernel<<<1, 32, 0, st>>>(sc);
  return cudaGetLastError();
}

cudaError_t launch_prim(const GridDev& G, const double* src, int src_prim, size_t plane, double phifac, double* out,
                        double* p_out, double gm1, bool mag, bool glm, int nblocks, cudaStream_t st) {
  if (mag && glm)
    prim_kernel<true, true><<<nblocks, 256, 0, st>>>(G, src, src_prim, plane, phifac, out, p_out, gm1);
  else if (mag)
    prim_kernel<true, false><<<nblocks, 256, 0, st>>>(G, src, src_prim, plane, phifac, out, p_out, gm1);
  else
    prim_kernel<false, false><<<nblocks, 256, 0, st>>>(G, src, src_prim, plane, phifac, out, p_out, gm1);
  return cudaGetLastError();
}

}  // namespace hmn

// ---------------------------------------------------------------------------
// Hyperbolic self-gravity (gravity_hyperbolic.f90:61-125, 230-280) with a
// Cartesian 7-point Laplacian: the counterpart of the 3-D spherical
// coefficients of gravity_hyperbolic.f90:385-406 with unit radial weights;
// each non-periodic face carries the Robin condition phi ~ 1/r folded into
// the centre coefficient as gravity_hyperbolic.f90:400-404 does.

namespace hmn {

__device__ __forceinline__ double rdist(const GridDev& G, int i, int j, int k) {
  const double x = G.g[0].x[i + 2], y = G.g[1].x[j + 2], z = G.g[2].x[k + 2];
  return sqrt(x * x + y * y + z * z);
}

__global__ void __launch_bounds__(256) hg_stage_kernel(const GridDev G, const HGArgs A) {
  const size_t plane = A.plane;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < plane; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % G.n[0]);
    const int j = (int)((c / G.n[0]) % G.n[1]);
    const int k = (int)(c / ((size_t)G.n[0] * G.n[1]));
    const AxisGeo &gx = G.g[0], &gy = G.g[1], &gz = G.g[2];
    double c0 = -((gx.idx[i + 2] + gx.idx[i + 3]) * gy.dxi[j + 2] * gz.dxi[k + 2] +
                  (gy.idx[j + 2] + gy.idx[j + 3]) * gx.dxi[i + 2] * gz.dxi[k + 2] +
                  (gz.idx[k + 2] + gz.idx[k + 3]) * gx.dxi[i + 2] * gy.dxi[j + 2]);
    double cm[3], cp[3];
    cm[0] = gy.dxi[j + 2] * gz.dxi[k + 2] / gx.dx[i + 2];
    cp[0] = gy.dxi[j + 2] * gz.dxi[k + 2] / gx.dx[i + 3];
    cm[1] = gx.dxi[i + 2] * gz.dxi[k + 2] / gy.dx[j + 2];
    cp[1] = gx.dxi[i + 2] * gz.dxi[k + 2] / gy.dx[j + 3];
    cm[2] = gx.dxi[i + 2] * gy.dxi[j + 2] / gz.dx[k + 2];
    cp[2] = gx.dxi[i + 2] * gy.dxi[j + 2] / gz.dx[k + 3];
    const int ijk[3] = {i, j, k};
    bool use_m[3] = {true, true, true}, use_p[3] = {true, true, true};
    size_t nbm[3], nbp[3];
    for (int a = 0; a < 3; a++) {
      const int n = G.n[a];
      const bool per = G.bc[a][0][0] == 0;
      int m[3] = {i, j, k}, p[3] = {i, j, k};
      m[a] = ijk[a] - 1;
      p[a] = ijk[a] + 1;
      if (per) {
        if (m[a] < 0) m[a] += n;
        if (p[a] >= n) p[a] -= n;
      } else {
        if (ijk[a] == n - 1) {
          c0 = c0 + cp[a] * rdist(G, i, j, k) / rdist(G, p[0], p[1], p[2]);
          use_p[a] = false;
        }
        if (ijk[a] == 0) {
          c0 = c0 + cm[a] * rdist(G, i, j, k) / rdist(G, m[0], m[1], m[2]);
          use_m[a] = false;
        }
      }
      nbm[a] = use_m[a] ? cidx(G, m[0], m[1], m[2]) : c;
      nbp[a] = use_p[a] ? cidx(G, p[0], p[1], p[2]) : c;
    }
    const double cn = gx.dxi[i + 2] * gy.dxi[j + 2] * gz.dxi[k + 2];
    const double* ph = A.phi_in;
    double lap = c0 * ph[c];
    for (int a = 0; a < 3; a++) {
      if (use_m[a]) lap = lap + cm[a] * ph[nbm[a]];
      if (use_p[a]) lap = lap + cp[a] * ph[nbp[a]];
    }
    const double lapphi = lap / cn;
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
  hg_stage_kernel<<<nblocks, 256, 0, st>>>(G, A);
  return cudaGetLastError();
}

}  // namespace hmn
