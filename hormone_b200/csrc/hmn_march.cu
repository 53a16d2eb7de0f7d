// hmn_march.cu -- the FP64 RK stage of a 3-D Cartesian grid as a march
// along z.
//
// A CTA owns a column of TX x TY cells in x-y and LZ planes in z.  It walks
// the planes bottom to top, keeping a rolling window of three staged planes
// in shared memory, and per plane k it:
//   phase 1: computes, per column, the z slope of plane k+1 (one owner
//            thread per column) and the x and y limited slopes of plane k
//            (all threads);
//   phase 2: computes, per column, the z face flux k+1/2 and the z flux
//            difference of cell k (owners, first), and the x and y HLLD face
//            fluxes of plane k (all threads);
//   phase 3: applies the RK combination, the source and the primitive
//            recovery to cell k of every column and writes U and P (owners),
//            while the other threads stage plane k+3 into the slot plane k
//            frees.
// The arithmetic of every slope, face and cell is that of the tile kernel
// (hmn_kernels.cu: axis_pass, stage_tile_exact), so the result is bitwise
// the same: interpolation.f90:15-490 (slopes, eint check), numflux.f90:46-218
// (face states), hlldflux.f90:19-179 (HLLD), rungekutta.f90:35-59 (update),
// source.f90:70-85 (gravity), rungekutta.f90:205-229 (primitives).
//
// Why a march: a z slope and a z face are computed once per cell instead of
// 10/8 and 9/8 times for an 8x8x8 tile; each plane is staged once per column
// tile instead of a cross-shaped 8x8x8 region (1,280 cells per 512); and the
// shared memory (108 KB: three 16x8 planes with their x-y halo, x-y slopes
// and fluxes of one plane, the z slopes and fluxes of one plane) lets two
// CTAs share an SM, so one CTA's barrier waits overlap the other's work.
// The z quantities of a column never leave the thread that owns it: its z
// slope crosses one barrier in registers and then waits in shared memory for
// the next plane, its z flux waits in shared memory, and the z flux
// difference is applied by the same thread in phase 3.
//
// Quotients: the stage is bound by the issue of dependent FP64 instructions,
// and about 190 of them per cell are IEEE divisions, most sharing a
// denominator with others (per face, 35 quotients have 11 denominators).
// Slopes, faces and the primitive recovery form them with FastDiv
// (hmn_div.cuh): one correctly rounded reciprocal per denominator, then a
// branch-free two-step correction per quotient, which yields the IEEE
// quotient bit for bit; where an operand lies outside the range in which
// that holds, the slope, face or cell is recomputed with IEEE division.
#include <cuda_runtime.h>

#include <cstdlib>

#include "hmn_div.cuh"
#include "hmn_face.cuh"
#include "hmn_internal.h"
#include "hmn_math.cuh"
#include "hmn_tile.cuh"

namespace hmn {
namespace {

// TX x TY columns (one owner thread each), NH more threads, MINB resident
// CTAs per SM.  OXY: the owners also take x-y slope and face items (the last
// NC of each list), for tiles whose other threads are fewer than the items.
template <int TX_, int TY_, int NH_, int MINB_, bool OXY_>
struct March {
  static constexpr int TX = TX_, TY = TY_, NC = TX * TY, NH = NH_, NT = NC + NH, MINB = MINB_;
  static constexpr bool OXY = OXY_;
  // staged cells of one plane: rows j in [0, TY) extended by two cells in x,
  // then the two rows below the tile and the two above (no corners)
  static constexpr int NROW = (TX + 4) * TY;
  static constexpr int NPL = NROW + 4 * TX;
  static constexpr int NSX = (TX + 2) * TY, NSY = TX * (TY + 2), NSXY = NSX + NSY;  // x, y slope cells
  static constexpr int NFX = (TX + 1) * TY, NFY = TX * (TY + 1), NFXY = NFX + NFY;  // x, y faces
  __device__ static __forceinline__ int pidx(int i, int j) {
    if (j < 0) return NROW + (j + 2) * TX + i;
    if (j >= TY) return NROW + 2 * TX + (j - TY) * TX + i;
    return j * (TX + 4) + i + 2;
  }
  __device__ static __forceinline__ void cell_of(int w, int& i, int& j) {
    if (w < NROW) {
      i = w % (TX + 4) - 2;
      j = w / (TX + 4);
    } else {
      const int v = w - NROW, r = v / TX;
      i = v % TX;
      j = r < 2 ? r - 2 : TY + r - 2;
    }
  }
};

template <class MT>
struct MarchSmem {
  double W[3][NQ][MT::NPL];    // rolling window: plane p in slot (p - k0 + 2) % 3
  double S[NS][MT::NSXY];      // x slopes ((TX+2) x TY), then y slopes (TX x (TY+2)) of plane k
  double F[9][MT::NFXY];       // x faces ((TX+1) x TY), then y faces (TX x (TY+1)) of plane k
  double SZ[NS][MT::NC];       // per column: the z slope of plane k
  double FZ[9][MT::NC];        // per column: the z flux through face k-1/2
};

// Stage plane p into window slot W (cells first, first + stride, ...): every
// cell of the tile's columns and, with `ring`, the two cells beyond each x
// and y face of the tile.  Cells outside the grid come from the boundary
// codes (stage_cell); of a plane outside the grid in z only the columns are
// needed (it is never swept in x or y).
template <bool MAG, bool GLM, class MT>
__device__ __forceinline__ void stage_plane(const GridDev& G, const StageArgs& A, double (*W)[MT::NPL], int p,
                                            bool ring, int x0, int y0, int T0, int T1, int first, int stride) {
  for (int w = first; w < MT::NPL; w += stride) {
    int i, j;
    MT::cell_of(w, i, j);
    const bool col = i >= 0 && i < T0 && j >= 0 && j < T1;
    if (!col) {
      if (!ring) continue;
      const bool xr = i >= -2 && i < T0 + 2 && j >= 0 && j < T1;
      const bool yr = i >= 0 && i < T0 && j >= -2 && j < T1 + 2;
      if (!xr && !yr) continue;
    }
    double q[NQ];
    stage_cell<MAG, GLM>(G, A, x0 + i, y0 + j, p, q);
#pragma unroll
    for (int s = 0; s < NQ; s++) W[s][w] = q[s];
  }
}

// The Cartesian gravity source of cell c (source.f90:70-85 with the centred
// force of get_fieldforce, source.f90:177-228), added to acc[1..4] as the
// tile kernel adds it.
__device__ __forceinline__ void cart_gravity(const GridDev& G, const StageArgs& A, size_t c, int i, int j, int k,
                                             double acc[9]) {
  const size_t pl = A.plane;
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
      } else if (a == 2 && G.ghalo[o > 0] != nullptr) {
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

// z flux of the face above the column's cell (k+1/2) from the window: the
// left state from plane k with the z slope the column keeps in SZ, the
// right one from plane k+1 with its slope in the thread's array sr (which
// the slope call filled in place: it is handed on, not copied).  The flux
// lands in fz already rotated into the conserved slots (put_flux with unit
// stride; numflux.f90:531-543).
template <bool MAG, class MT>
__device__ __forceinline__ bool z_face(const double* Wk, const double* Wk1, const MarchSmem<MT>& sm, int t,
                                       const double* sr, const AxisGeo& gz, int k, const StageArgs& A, double ch,
                                       double fz[9]) {
  constexpr int QS = MT::NPL;
  const double dx1 = gz.hr[k + 2], dx2 = gz.hl[k + 3];
  return face_flux_fast<MAG, QS>(Wk, Wk1, &sm.SZ[0][t], MT::NC, sr, 1, dx1, dx2, 2, 0, 1, A.gamma, A.gm1, ch, fz, 1);
}

// Ask for the line of p to be brought into L2 (no register, no wait).
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.L2 [%0];" ::"l"(p)); }

template <bool MAG, bool GLM, int LIM, class MT, bool PUSH>
__global__ void __launch_bounds__(MT::NT, MT::MINB)
    march_stage_kernel(const __grid_constant__ GridDev G, const __grid_constant__ StageArgs A, int LZ, int ntx,
                       int nty) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  MarchSmem<MT>& sm = *reinterpret_cast<MarchSmem<MT>*>(smem_raw);
  if (A.sc->done) return;
  constexpr int TX = MT::TX, TY = MT::TY, NC = MT::NC, NH = MT::NH, NT = MT::NT, QS = MT::NPL;
  constexpr int nv = MAG ? (GLM ? 9 : 8) : 5;
  const int tid = threadIdx.x;
  int b = blockIdx.x;
  const int x0 = (b % ntx) * TX;
  b /= ntx;
  const int y0 = (b % nty) * TY;
  const int k0 = (b / nty) * LZ;
  const int T0 = min(TX, G.n[0] - x0), T1 = min(TY, G.n[1] - y0);
  const int kend = min(k0 + LZ, G.n[2]);
  const double ch = A.sc->ch;
  const AxisGeo& gz = G.g[2];
  auto slot = [&](int p) { return (p - k0 + 2) % 3; };

  // owner threads: one column each
  const bool owner = tid < NC;
  const int oi = tid % TX, oj = tid / TX;
  const bool live = owner && oi < T0 && oj < T1;
  const int orr = MT::pidx(oi, oj);
  const int h = tid - NC;  // index of the other threads

  // ---- prologue: planes k0-2 .. k0+2, the z slopes of k0-1 and k0, face k0-1/2
  for (int p = k0 - 2; p <= k0; p++)
    stage_plane<MAG, GLM, MT>(G, A, sm.W[slot(p)], p, p >= k0 && p < kend, x0, y0, T0, T1, tid, NT);
  __syncthreads();
  double szn[NS];  // the z slope of the plane above the one being finished
  if (live)
    slopes_to<MAG, LIM, QS>(&sm.W[slot(k0 - 2)][0][orr], &sm.W[slot(k0 - 1)][0][orr], &sm.W[slot(k0)][0][orr], gz,
                            k0 - 1, szn, 1);
  __syncthreads();
  stage_plane<MAG, GLM, MT>(G, A, sm.W[slot(k0 + 1)], k0 + 1, k0 + 1 < kend, x0, y0, T0, T1, tid, NT);
  __syncthreads();
  if (live) {
#pragma unroll
    for (int q = 0; q < NS; q++) sm.SZ[q][tid] = szn[q];  // the slope of k0-1 is the face's left slope
    double szk[NS];
    slopes_to<MAG, LIM, QS>(&sm.W[slot(k0 - 1)][0][orr], &sm.W[slot(k0)][0][orr], &sm.W[slot(k0 + 1)][0][orr], gz,
                            k0, szk, 1);
    double fz[9];
    if (!z_face<MAG, MT>(&sm.W[slot(k0 - 1)][0][orr], &sm.W[slot(k0)][0][orr], sm, tid, szk, gz, k0 - 1, A, ch, fz))
      record_error(A.sc, kENEG_EINT, x0 + oi, y0 + oj, k0 - 1);
    if (k0 == 0 && G.fb != nullptr) {  // boundary code 10 at the inner z face (fluxboundary.f90:42-87)
#pragma unroll
      for (int q = 0; q < 9; q++) fz[q] = G.fb[q];
    }
#pragma unroll
    for (int q = 0; q < NS; q++) sm.SZ[q][tid] = szk[q];
#pragma unroll
    for (int q = 0; q < 9; q++) sm.FZ[q][tid] = fz[q];
  }
  __syncthreads();
  stage_plane<MAG, GLM, MT>(G, A, sm.W[slot(k0 + 2)], k0 + 2, k0 + 2 < kend, x0, y0, T0, T1, tid, NT);
  __syncthreads();

  const size_t pl = A.plane;
  const double dtf = A.fact * A.sc->dt;
  for (int k = k0; k < kend; k++) {
    const double* Wk = &sm.W[slot(k)][0][0];
    const double* Wk1 = &sm.W[slot(k + 1)][0][0];
    const double* Wk2 = &sm.W[slot(k + 2)][0][0];
    // ---- prefetch into L2 what phase 3 reads from HBM: the owners' U of
    // cell k, the other threads' cells of plane k+3 (interior cells only)
    if (live) {
      const size_t c = cidx(G, x0 + oi, y0 + oj, k);
#pragma unroll
      for (int q = 0; q < nv; q++) {
        prefetch_l2(A.uorg + q * pl + c);
        if (A.ucur != A.uorg) prefetch_l2(A.ucur + q * pl + c);
      }
    } else if (!owner && k + 3 <= kend + 1 && k + 3 < G.n[2]) {
      for (int w = h; w < MT::NPL; w += NH) {
        int i, j;
        MT::cell_of(w, i, j);
        const int gi = x0 + i, gj = y0 + j;
        const bool col = i >= 0 && i < T0 && j >= 0 && j < T1;
        const bool ring = k + 3 < kend && ((i >= -2 && i < T0 + 2 && j >= 0 && j < T1) ||
                                           (i >= 0 && i < T0 && j >= -2 && j < T1 + 2));
        if (!(col || ring) || gi < 0 || gi >= G.n[0] || gj < 0 || gj >= G.n[1]) continue;
        const size_t c = cidx(G, gi, gj, k + 3);
#pragma unroll
        for (int q = 0; q < NP; q++) prefetch_l2(A.pin + q * pl + c);
      }
    }
    // ---- phase 1: slopes --------------------------------------------------------
    // owners: the z slope of their column, then one x-y slope cell each (the
    // last NC of the list); the other threads: the rest of the list
    if (live) slopes_to<MAG, LIM, QS>(Wk + orr, Wk1 + orr, Wk2 + orr, gz, k + 1, szn, 1);
    constexpr int NSO = MT::OXY ? MT::NSXY - NC : MT::NSXY;  // items the other threads take
    for (int w = owner ? (MT::OXY ? NSO + tid : MT::NSXY) : h; w < (owner ? MT::NSXY : NSO);
         w += owner ? NC : NH) {
      int ax, si, sj;
      if (w < MT::NSX) {
        ax = 0;
        si = w % (TX + 2) - 1;
        sj = w / (TX + 2);
        if (si > T0 || sj >= T1) continue;
      } else {
        ax = 1;
        si = (w - MT::NSX) % TX;
        sj = (w - MT::NSX) / TX - 1;
        if (si >= T0 || sj > T1) continue;
      }
      const int r = MT::pidx(si, sj);
      const int rm = ax == 0 ? MT::pidx(si - 1, sj) : MT::pidx(si, sj - 1);
      const int rp = ax == 0 ? MT::pidx(si + 1, sj) : MT::pidx(si, sj + 1);
      slopes_to<MAG, LIM, QS>(Wk + rm, Wk + r, Wk + rp, G.g[ax], ax == 0 ? x0 + si : y0 + sj, &sm.S[0][w],
                              MT::NSXY);
    }
    __syncthreads();
    // ---- phase 2: face fluxes -------------------------------------------------
    // owners: first the z face of their column (its slopes are at hand, and
    // the z flux difference is then done before the x-y face call)
    double dz[9];
    if (live) {
      double fz[9];
      if (!z_face<MAG, MT>(Wk + orr, Wk1 + orr, sm, tid, szn, gz, k, A, ch, fz))
        record_error(A.sc, kENEG_EINT, x0 + oi, y0 + oj, k);
      const double idz = gz.idxi[k + 2];
#pragma unroll
      for (int q = 0; q < 9; q++) {
        dz[q] = idz * (sm.FZ[q][tid] - fz[q]);
        sm.FZ[q][tid] = fz[q];
      }
#pragma unroll
      for (int q = 0; q < NS; q++) sm.SZ[q][tid] = szn[q];
    }
    // owners, then: one x-y face each (the last NC of the list); the other
    // threads: the rest of the list
    constexpr int NFO = MT::OXY ? MT::NFXY - NC : MT::NFXY;
    for (int w = owner ? (MT::OXY ? NFO + tid : MT::NFXY) : h; w < (owner ? MT::NFXY : NFO);
         w += owner ? NC : NH) {
      int ax, fi, fj, sL, sR, rL, rR, gL;
      if (w < MT::NFX) {
        ax = 0;
        const int f = w % (TX + 1);
        fj = w / (TX + 1);
        if (f > T0 || fj >= T1) continue;
        fi = f;
        rL = MT::pidx(f - 1, fj);
        rR = MT::pidx(f, fj);
        sL = f + (TX + 2) * fj;
        sR = sL + 1;
        gL = x0 + f - 1;
      } else {
        ax = 1;
        fi = (w - MT::NFX) % TX;
        const int f = (w - MT::NFX) / TX;
        if (fi >= T0 || f > T1) continue;
        fj = f;
        rL = MT::pidx(fi, f - 1);
        rR = MT::pidx(fi, f);
        sL = MT::NSX + fi + TX * f;
        sR = sL + TX;
        gL = y0 + f - 1;
      }
      const AxisGeo& g = G.g[ax];
      const double dx1 = g.hr[gL + 2], dx2 = g.hl[gL + 3];
      const int cn = ax, c1 = ax + 1, c2 = (ax + 2) % 3;
      const double* PL = Wk + rL;
      const double* PR = Wk + rR;
      const double* SLp = &sm.S[0][sL];
      const double* SRp = &sm.S[0][sR];
      constexpr int SS = MT::NSXY;
      // the flux goes straight into its conserved slots of F (put_flux)
      if (!face_flux_fast<MAG, QS>(PL, PR, SLp, SS, SRp, SS, dx1, dx2, cn, c1, c2, A.gamma, A.gm1, ch, &sm.F[0][w],
                                   MT::NFXY)) {
        int gi[3] = {x0 + fi, y0 + fj, k};
        gi[ax] = gL;
        record_error(A.sc, kENEG_EINT, gi[0], gi[1], gi[2]);
      }
    }
    __syncthreads();
    // ---- phase 3: cell update (owners), staging of plane k+3 (the others) -------
    if (owner) {
      if (live) {
        const int i = x0 + oi, j = y0 + oj;
        const size_t c = cidx(G, i, j, k);
        double acc[9];
        const double idx1 = G.g[0].idxi[i + 2], idx2 = G.g[1].idxi[j + 2];
        const int xm = oi + (TX + 1) * oj, ym = MT::NFX + oi + TX * oj;
#pragma unroll
        for (int q = 0; q < nv; q++) {
          acc[q] = 0.0;
          acc[q] = acc[q] + idx1 * (sm.F[q][xm] - sm.F[q][xm + 1]);
          acc[q] = acc[q] + idx2 * (sm.F[q][ym] - sm.F[q][ym + TX]);
          acc[q] = acc[q] + dz[q];
        }
        if (A.gphi != nullptr) cart_gravity(G, A, c, i, j, k, acc);
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
        if constexpr (PUSH) push_boundary_layers(G, A, Po, c, i, j, k);
      }
    } else if (k + 3 <= kend + 1) {
      // plane k+3 into the slot plane k leaves (last read in phase 2)
      stage_plane<MAG, GLM, MT>(G, A, sm.W[slot(k + 3)], k + 3, k + 3 < kend, x0, y0, T0, T1, h, NH);
    }
    __syncthreads();
  }
}

// 16x8 columns with 128 more threads; the owners take x-y items too, so
// every thread has one to two items per phase
using MT168 = March<16, 8, 128, 2, true>;

template <bool MAG, bool GLM, int LIM, bool PUSH, class MT>
cudaError_t launch_mt(const GridDev& G, const StageArgs& A, int LZ, int ntx, int nty, int nch, cudaStream_t st) {
  constexpr int smem = (int)sizeof(MarchSmem<MT>);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(march_stage_kernel<MAG, GLM, LIM, MT, PUSH>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(march_stage_kernel<MAG, GLM, LIM, MT, PUSH>,
                             cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  march_stage_kernel<MAG, GLM, LIM, MT, PUSH><<<ntx * nty * nch, MT::NT, smem, st>>>(G, A, LZ, ntx, nty);
  return cudaGetLastError();
}

template <bool MAG, bool GLM, int LIM, bool PUSH>
cudaError_t launch_t(const GridDev& G, const StageArgs& A, int LZ, int ntx, int nty, int nch, cudaStream_t st) {
  return launch_mt<MAG, GLM, LIM, PUSH, MT168>(G, A, LZ, ntx, nty, nch, st);
}

template <bool MAG, bool GLM, bool PUSH>
cudaError_t launch_lim(const GridDev& G, const StageArgs& A, int LZ, int ntx, int nty, int nch, cudaStream_t st) {
  if (A.limiter == 0) return launch_t<MAG, GLM, 0, PUSH>(G, A, LZ, ntx, nty, nch, st);
  if (A.limiter == 1) return launch_t<MAG, GLM, 1, PUSH>(G, A, LZ, ntx, nty, nch, st);
  return launch_t<MAG, GLM, 2, PUSH>(G, A, LZ, ntx, nty, nch, st);
}

template <bool PUSH>
cudaError_t launch_mag(const GridDev& G, const StageArgs& A, bool mag, bool glm, int LZ, int ntx, int nty, int nch,
                       cudaStream_t st) {
  if (mag && glm) return launch_lim<true, true, PUSH>(G, A, LZ, ntx, nty, nch, st);
  if (mag) return launch_lim<true, false, PUSH>(G, A, LZ, ntx, nty, nch, st);
  return launch_lim<false, false, PUSH>(G, A, LZ, ntx, nty, nch, st);
}

int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
  }
  return n;
}

}  // namespace

// HMN_MARCH=0 keeps 3-D Cartesian grids on the tile kernel (read at every
// launch; a captured CUDA graph keeps the kernel it was captured with)
bool march_enabled() {
  const char* e = getenv("HMN_MARCH");
  return !(e && e[0] == '0');
}

void march_chunks(const int n[3], int* lz, int* ntx, int* nty, int* nch) {
  *ntx = (n[0] + MT168::TX - 1) / MT168::TX;
  *nty = (n[1] + MT168::TY - 1) / MT168::TY;
  // z chunks: about twelve CTAs per SM in all (six waves of two), each chunk at least 16 planes
  const long long cols = (long long)(*ntx) * (*nty);
  long long want = (12LL * sm_count() + cols - 1) / cols;
  if (want < 1) want = 1;
  int l = (int)((n[2] + want - 1) / want);
  if (l < 16) l = 16;
  if (l > n[2]) l = n[2];
  *lz = l;
  *nch = (n[2] + l - 1) / l;
}

cudaError_t launch_stage_march(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st) {
  if (!march_enabled() || G.sph.on || A.nspc > 0 || !(G.solve[0] && G.solve[1] && G.solve[2]))
    return cudaErrorNotSupported;
  int lz, ntx, nty, nch;
  const bool push = A.push[0] != nullptr || A.push[1] != nullptr;
  march_chunks(G.n, &lz, &ntx, &nty, &nch);
  if (push) return launch_mag<true>(G, A, mag, glm, lz, ntx, nty, nch, st);
  return launch_mag<false>(G, A, mag, glm, lz, ntx, nty, nch, st);
}

}  // namespace hmn
