// hmn_tile.cuh -- tile geometry and ghost-cell staging shared by the FP64
// and the mixed-precision stage kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "hmn_internal.h"
#include "hmn_math.cuh"
#include "hmn_tma.cuh"

namespace hmn {

// conserved slots (checksetup.f90:61-75)
enum { ICNT = 0, IMO1 = 1, IENE = 4, IMG1 = 5, I9WV = 8 };
// primitive planes in HBM
enum { PD = 0, PV = 1, PE = 4, PB = 5, PPHI = 8, PEINT = 9, NP = 10 };
// staged quantities per cell in shared memory: d, m1..3 (= d*v), e, b1..3, phi, eint
enum { Q_D = 0, Q_M = 1, Q_E = 4, Q_B = 5, Q_PHI = 8, Q_EINT = 9, NQ = 10 };
// slopes: d, e, m1..3, b1..3
enum { S_D = 0, S_E = 1, S_M = 2, S_B = 5, NS = 8 };


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

// Compile-time description of a tile: TX x TY x TZ cells (256 in all) and a
// halo of two cells beyond each face of every axis with extent > 1.
template <int TX_, int TY_, int TZ_, int NT_ = 256, int MINB_ = 2, int SP_ = 0>
struct Tile {
  static constexpr int TX = TX_, TY = TY_, TZ = TZ_;
  static constexpr int SP = SP_;      // passive scalars the shared-memory layout has room for
  // threads per CTA: at least the tile's cell count, and best the size of the
  // largest per-axis slope box, so that every phase of an axis pass takes one
  // round (16x16 -> 288, 256 -> 288, 32x8 -> 320, 8x8x4 -> 384, 8x8x8 -> 640)
  static constexpr int NT = NT_;
  static constexpr int MINB = MINB_;  // resident CTAs per SM the register budget is sized for
  static constexpr int NC = TX * TY * TZ;
  static constexpr int HX = TX > 1 ? 2 : 0, HY = TY > 1 ? 2 : 0, HZ = TZ > 1 ? 2 : 0;
  // region part 0: x-extended rows of every interior (j,k); part 1: y halos; part 2: z halos
  static constexpr int N0 = (TX + 2 * HX) * TY * TZ;
  static constexpr int N1 = TX * (2 * HY) * TZ;
  static constexpr int N2 = TX * TY * (2 * HZ);
  static constexpr int NR = N0 + N1 + N2;
  static constexpr int maxi(int a, int b) { return a > b ? a : b; }
  // slope and face boxes of the largest solved axis (axes of extent 1 are never swept)
  static constexpr int NSB = maxi(maxi(HX ? (TX + 2) * TY * TZ : 1, HY ? TX * (TY + 2) * TZ : 1),
                                  HZ ? TX * TY * (TZ + 2) : 1);
  static constexpr int NFB = maxi(maxi(HX ? (TX + 1) * TY * TZ : 1, HY ? TX * (TY + 1) * TZ : 1),
                                  HZ ? TX * TY * (TZ + 1) : 1);
  // shared-memory slot of local cell (i,j,k); at most one coordinate lies outside the tile.
  // Part 1 holds the low y halo (TX x 2 x TZ, x fastest) and then the high one, part 2 the
  // low and then the high z halo (TX x TY x 2): each is one box of the 4-D plane tensor.
  __device__ static __forceinline__ int pidx(int i, int j, int k) {
    if (HY && (j < 0 || j >= TY)) {
      const int hi = j < 0 ? 0 : 1;
      const int jl = j < 0 ? j + 2 : j - TY;
      return N0 + hi * (N1 / 2) + i + TX * (jl + 2 * k);
    }
    if (HZ && (k < 0 || k >= TZ)) {
      const int kk = k < 0 ? k + 2 : k - TZ + 2;
      return N0 + N1 + i + TX * (j + TY * kk);
    }
    return (i + HX) + (TX + 2 * HX) * (j + TY * k);
  }
  // local cell of region slot w
  __device__ static __forceinline__ void region_cell(int w, int& i, int& j, int& k) {
    if (w < N0) {
      constexpr int RX = TX + 2 * HX;
      i = w % RX - HX;
      j = (w / RX) % TY;
      k = w / (RX * TY);
    } else if (w < N0 + N1) {
      constexpr int H1 = N1 > 0 ? N1 / 2 : 1;  // one y halo (only reached when there are y halos)
      const int v = w - N0;
      const int hi = v / H1, r = v % H1;
      i = r % TX;
      const int jl = (r / TX) % 2;
      k = r / (TX * 2);
      j = hi ? TY + jl : jl - 2;
    } else {
      const int v = w - N0 - N1;
      i = v % TX;
      j = (v / TX) % TY;
      const int kk = v / (TX * TY);
      k = kk < 2 ? kk - 2 : TZ + kk - 2;
    }
  }
};

// Staged quantities of a global cell (i,j,k): interior cells from P, ghost
// cells (one axis out of range) through the boundary codes.
template <bool MAG, bool GLM>
__device__ __forceinline__ void stage_cell(const GridDev& G, const StageArgs& A, int i, int j, int k,
                                           double* q /* NQ values */) {
  const double* P = A.pin;
  const size_t pl = A.plane;
  int c3[3] = {i, j, k};
  int ax = -1;
#pragma unroll
  for (int a = 0; a < 3; a++)
    if (c3[a] < 0 || c3[a] >= G.n[a]) ax = a;
  if (ax < 0) {
    const size_t c = cidx(G, i, j, k);
    const double d = P[c];
    q[Q_D] = d;
    q[Q_M + 0] = d * P[PV * pl + c];
    q[Q_M + 1] = d * P[(PV + 1) * pl + c];
    q[Q_M + 2] = d * P[(PV + 2) * pl + c];
    q[Q_E] = P[PE * pl + c];
    if (MAG) {
      q[Q_B + 0] = P[PB * pl + c];
      q[Q_B + 1] = P[(PB + 1) * pl + c];
      q[Q_B + 2] = P[(PB + 2) * pl + c];
    } else {
      q[Q_B + 0] = q[Q_B + 1] = q[Q_B + 2] = 0.0;
    }
    q[Q_PHI] = GLM ? P[PPHI * pl + c] * A.phifac : 0.0;
    q[Q_EINT] = P[PEINT * pl + c];
    return;
  }
  const int n = G.n[ax];
  const int s = c3[ax];
  const int io = s < 0 ? 0 : 1;
  const int gl = io == 0 ? s + 2 : s - n;  // ghost layer 0 or 1
  if (ax == 2 && G.zhalo[io] != nullptr) {
    // a neighbouring slab's interior cell: staged exactly as our own interior cells
    const size_t hp = (size_t)G.n[0] * G.n[1];
    const size_t h = (size_t)gl * hp + (size_t)i + (size_t)G.n[0] * j;
    const double* H = G.zhalo[io];
    const double d = H[h];
    const double v1 = H[PV * 2 * hp + h], v2 = H[(PV + 1) * 2 * hp + h], v3 = H[(PV + 2) * 2 * hp + h];
    const double b1 = MAG ? H[PB * 2 * hp + h] : 0.0, b2 = MAG ? H[(PB + 1) * 2 * hp + h] : 0.0;
    const double b3 = MAG ? H[(PB + 2) * 2 * hp + h] : 0.0;
    q[Q_D] = d;
    q[Q_M + 0] = d * v1;
    q[Q_M + 1] = d * v2;
    q[Q_M + 2] = d * v3;
    q[Q_B + 0] = b1;
    q[Q_B + 1] = b2;
    q[Q_B + 2] = b3;
    q[Q_PHI] = GLM ? H[PPHI * 2 * hp + h] * A.phifac : 0.0;
    if (G.zwrap[io]) {  // periodic ghost as the boundary condition forms it (see below)
      const double eg = (A.gm1 * H[PEINT * 2 * hp + h]) / A.gm1;
      q[Q_E] = eg + 0.5 * (d * (v1 * v1 + v2 * v2 + v3 * v3) + b1 * b1 + b2 * b2 + b3 * b3);
      q[Q_EINT] = eg;
    } else {
      q[Q_E] = H[PE * 2 * hp + h];
      q[Q_EINT] = H[PEINT * 2 * hp + h];
    }
    return;
  }
  const int per = io == 0 ? n - 2 + gl : gl;
  const int refl = io == 0 ? 1 - gl : n - 1 - gl;
  const int edge = io == 0 ? 0 : n - 1;
  const int bs = G.bc[ax][io][0], bv = G.bc[ax][io][1];
  c3[ax] = bs == 0 ? per : (bs == 1 ? refl : edge);
  const size_t cs = cidx(G, c3[0], c3[1], c3[2]);  // scalar image (d, p, phi); the edge cell for 4/5/9
  c3[ax] = bv == 0 ? per : (bv == 1 ? refl : edge);
  const size_t cv = cidx(G, c3[0], c3[1], c3[2]);  // vector image (v, B); the edge cell for 4/5/9
  c3[ax] = io == 0 ? 1 : n - 2;
  const size_t cin = cidx(G, c3[0], c3[1], c3[2]);  // the cell next to the edge cell, inward
  // linear extrapolation from the edge cell (codes 4/5, boundarycondition.f90:302-327,419-468,963-985):
  // both ghosts of the face, the near one from the interior and the far one from the near one
  const bool far = io == 0 ? gl == 0 : gl == 1;
  const double* dxa = G.g[ax].dx + 2;
  auto linear = [&](double f0, double f1, double& g0, double& g1) {
    if (io == 1) {
      g0 = f0 + (f0 - f1) * dxa[n - 1] / dxa[n - 2];
      g1 = g0 + (g0 - f0) * dxa[n] / dxa[n - 1];
    } else {
      g0 = f0 - (f1 - f0) * dxa[0] / dxa[1];
      g1 = g0 - (f0 - g0) * dxa[-1] / dxa[0];
    }
  };
  // Dirichlet values of this ghost (code 9; code 10 keeps the host's ghosts the
  // same way): 8 + nspc planes x 2 layers x face cells
  const double* D = G.dir[ax][io];
  const int oa0 = ax == 0 ? 1 : 0, oa1 = ax == 2 ? 1 : 2;
  const size_t area = (size_t)G.n[oa0] * G.n[oa1];
  const size_t hd = (size_t)gl * area + (size_t)c3[oa0] + (size_t)G.n[oa0] * c3[oa1];
  double dg, pg, phig;
  if (bs == 4 || bs == 5) {
    double g0, g1;
    linear(P[cs], P[cin], g0, g1);
    if (g1 <= 0.0) g0 = g1 = P[cs];
    dg = far ? g1 : g0;
    linear(A.gm1 * P[PEINT * pl + cs], A.gm1 * P[PEINT * pl + cin], g0, g1);
    if (g1 <= 0.0) g0 = g1 = A.gm1 * P[PEINT * pl + cs];
    pg = far ? g1 : g0;
    phig = GLM ? P[PPHI * pl + cs] * A.phifac : 0.0;
  } else if (bs == 9 || bs == 10) {
    dg = D[hd];
    pg = D[2 * area + hd];
    phig = 0.0;
  } else {
    dg = P[cs];
    pg = A.gm1 * P[PEINT * pl + cs];  // pressure of the image cell (eos.f90:256)
    phig = GLM ? P[PPHI * pl + cs] * A.phifac : 0.0;
  }
  double v[3], b[3] = {0.0, 0.0, 0.0};
  if (bv == 4 || bv == 5) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double g0, g1;
      linear(P[(PV + c) * pl + cv], P[(PV + c) * pl + cin], g0, g1);
      v[c] = far ? g1 : g0;
      if (MAG) {
        linear(P[(PB + c) * pl + cv], P[(PB + c) * pl + cin], g0, g1);
        b[c] = far ? g1 : g0;
      }
    }
    if (bv == 5) {  // linear + outgoing: the normal velocity only flows out
      const double vedge = P[(PV + ax) * pl + cv];
      v[ax] = v[ax] * (io == 1 ? 0.5 + fsign(0.5, vedge) : 0.5 - fsign(0.5, vedge));
    }
  } else if (bv == 9 || bv == 10) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      v[c] = D[(size_t)(2 + c) * 2 * area + hd];
      if (MAG) b[c] = D[(size_t)(5 + c) * 2 * area + hd];
    }
  } else {
    v[0] = P[PV * pl + cv];
    v[1] = P[(PV + 1) * pl + cv];
    v[2] = P[(PV + 2) * pl + cv];
    if (MAG) {
      b[0] = P[PB * pl + cv];
      b[1] = P[(PB + 1) * pl + cv];
      b[2] = P[(PB + 2) * pl + cv];
    }
    double vn = v[ax];
    if (bv == 1) {
      vn = -vn;
      b[ax] = -b[ax];
    } else if (bv == 2) {
      if (io == 0)
        vn = ax == 0 ? fmin2(0.0, vn) : vn * (0.5 - fsign(0.5, vn));  // :165 and the y/z plug form
      else
        vn = vn * (0.5 + fsign(0.5, vn));
    }
    v[ax] = vn;
  }
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

// Interior cell whose scalar values the cell (i,j,k) holds: itself, or for a
// ghost (one coordinate outside the grid) its image under the scalar
// boundary code (boundarycondition.f90: periodic, reflective, outgoing/free).
__device__ __forceinline__ size_t scalar_image(const GridDev& G, int i, int j, int k) {
  int c3[3] = {i, j, k};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int n = G.n[a], s = c3[a];
    if (s >= 0 && s < n) continue;
    const int io = s < 0 ? 0 : 1;
    const int gl = io == 0 ? s + 2 : s - n;
    const int per = io == 0 ? n - 2 + gl : gl;
    const int refl = io == 0 ? 1 - gl : n - 1 - gl;
    const int edge = io == 0 ? 0 : n - 1;
    const int bs = G.bc[a][io][0];
    c3[a] = bs == 0 ? per : (bs == 1 ? refl : edge);
  }
  return cidx(G, c3[0], c3[1], c3[2]);
}

// The Dirichlet values of a ghost cell's face (scalar code 9 or 10), or nullptr;
// with the cell's index in that face's 2 x n1 x n2 layout and the face area.
__device__ __forceinline__ int out_axis(const GridDev& G, int i, int j, int k) {
  return (i < 0 || i >= G.n[0]) ? 0 : ((j < 0 || j >= G.n[1]) ? 1 : ((k < 0 || k >= G.n[2]) ? 2 : -1));
}
__device__ __forceinline__ const double* dirichlet_face(const GridDev& G, int i, int j, int k) {
  const int ax = out_axis(G, i, j, k);
  if (ax < 0) return nullptr;
  const int c3[3] = {i, j, k};
  const int io = c3[ax] < 0 ? 0 : 1;
  return G.bc[ax][io][0] >= 9 ? G.dir[ax][io] : nullptr;
}
__device__ __forceinline__ size_t dirichlet_area(const GridDev& G, int i, int j, int k) {
  const int ax = out_axis(G, i, j, k);
  const int oa0 = ax == 0 ? 1 : 0, oa1 = ax == 2 ? 1 : 2;
  return (size_t)G.n[oa0] * G.n[oa1];
}
__device__ __forceinline__ size_t dirichlet_index(const GridDev& G, int i, int j, int k) {
  const int ax = out_axis(G, i, j, k);
  const int c3[3] = {i, j, k};
  const int oa0 = ax == 0 ? 1 : 0, oa1 = ax == 2 ? 1 : 2;
  const int s = c3[ax], n = G.n[ax];
  const int gl = s < 0 ? s + 2 : s - n;
  return (size_t)gl * G.n[oa0] * G.n[oa1] + (size_t)c3[oa0] + (size_t)G.n[oa0] * c3[oa1];
}

// Stage the tile's cross-shaped stencil region (tile origin t0, real extent
// T) into P[NQ][NR], ending with __syncthreads().  With tensor maps (3-D
// tiles) the cells inside the grid arrive by TMA as raw primitive planes and
// are converted in place exactly as stage_cell converts them (m = d*v,
// phi*phifac); ghost cells are then written by stage_cell from the boundary
// codes.  Without maps every slot is loaded by stage_cell.
template <bool MAG, bool GLM, class TL>
__device__ __forceinline__ void stage_region(const GridDev& G, const StageArgs& A, double (*P)[TL::NR],
                                             uint64_t* bar, const TmaMaps* tm, const int t0[3], const int T[3]) {
  constexpr int TT[3] = {TL::TX, TL::TY, TL::TZ};
  const int tid = threadIdx.x;
  const bool tma = tm != nullptr && TL::SP == 0;  // scalar planes are staged by plain loads
  if (tma) {
    if (tid == 0) {
      mbar_init(bar, 1);
      mbar_init_fence();
    }
    __syncthreads();
    if (tid == 0) {
      mbar_arrive_expect_tx(bar, (uint32_t)(NQ * TL::NR * sizeof(double)));
      // HBM plane p -> staged slot (d, v1..3 (made m below), e, b1..3, phi, eint)
      constexpr int dst[NP] = {Q_D, Q_M, Q_M + 1, Q_M + 2, Q_E, Q_B, Q_B + 1, Q_B + 2, Q_PHI, Q_EINT};
#pragma unroll
      for (int p = 0; p < NP; p++) {
        double* base = P[dst[p]];
        tma_load_4d(base, &tm->box[0], bar, t0[0] - 2, t0[1], t0[2], p);
        tma_load_4d(base + TL::N0, &tm->box[1], bar, t0[0], t0[1] - 2, t0[2], p);
        tma_load_4d(base + TL::N0 + TL::N1 / 2, &tm->box[1], bar, t0[0], t0[1] + TL::TY, t0[2], p);
        tma_load_4d(base + TL::N0 + TL::N1, &tm->box[2], bar, t0[0], t0[1], t0[2] - 2, p);
        tma_load_4d(base + TL::N0 + TL::N1 + TL::N2 / 2, &tm->box[2], bar, t0[0], t0[1], t0[2] + TL::TZ, p);
      }
    }
    if (!mbar_try_wait(bar, 0)) {
      const unsigned long long t_start = global_ns();
      while (!mbar_try_wait(bar, 0)) {
        if (global_ns() - t_start > kTmaWaitNs) {
          record_error(A.sc, kETIMEOUT, t0[0], t0[1], t0[2]);
          break;
        }
      }
    }
  }
  for (int w = tid; w < TL::NR; w += TL::NT) {
    int lc[3];
    TL::region_cell(w, lc[0], lc[1], lc[2]);
    int out = 0;
    bool need = true;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if (lc[a] < 0 || lc[a] >= T[a]) {
        out++;
        if (TT[a] == 1 || lc[a] < -2 || lc[a] > T[a] + 1) need = false;
      }
    }
    if (!need || out > 1) continue;
    const int gi = t0[0] + lc[0], gj = t0[1] + lc[1], gk = t0[2] + lc[2];
    const bool ghost = gi < 0 || gi >= G.n[0] || gj < 0 || gj >= G.n[1] || gk < 0 || gk >= G.n[2];
    if (tma && !ghost) {
      const double d = P[Q_D][w];
      P[Q_M + 0][w] = d * P[Q_M + 0][w];
      P[Q_M + 1][w] = d * P[Q_M + 1][w];
      P[Q_M + 2][w] = d * P[Q_M + 2][w];
      if (!MAG) P[Q_B + 0][w] = P[Q_B + 1][w] = P[Q_B + 2][w] = 0.0;
      P[Q_PHI][w] = GLM ? P[Q_PHI][w] * A.phifac : 0.0;
      continue;
    }
    double q[NQ];
    stage_cell<MAG, GLM>(G, A, gi, gj, gk, q);
#pragma unroll
    for (int s = 0; s < NQ; s++) P[s][w] = q[s];
    if constexpr (TL::SP > 0) {
      const int zio = gk < 0 ? 0 : 1;
      if ((gk < 0 || gk >= G.n[2]) && G.zhalo[zio] != nullptr) {  // neighbouring slab
        const size_t hp = (size_t)G.n[0] * G.n[1];
        const size_t h = (size_t)(zio == 0 ? gk + 2 : gk - G.n[2]) * hp + (size_t)gi + (size_t)G.n[0] * gj;
        for (int n = 0; n < A.nspc; n++) P[NQ + n][w] = G.zhalo[zio][(size_t)(NP + n) * 2 * hp + h];
      } else if (const double* D = dirichlet_face(G, gi, gj, gk)) {
        const size_t hd = dirichlet_index(G, gi, gj, gk);
        const size_t two_area = 2 * dirichlet_area(G, gi, gj, gk);
        for (int n = 0; n < A.nspc; n++) P[NQ + n][w] = D[(size_t)(8 + n) * two_area + hd];
      } else {
        const size_t cs = scalar_image(G, gi, gj, gk);
        for (int n = 0; n < A.nspc; n++) P[NQ + n][w] = A.pin[(size_t)(NP + n) * A.plane + cs];
      }
    }
  }
  __syncthreads();
}


// RK coefficients (faco, fact, facn) of stage `iter` of an rktype scheme
// (rungekutta.f90:146-183)
__host__ __device__ __forceinline__ void rk_coefficients(int iter, int type, double* faco, double* fact,
                                                         double* facn) {
  if (type == 3) {
    if (iter == 1) {
      *faco = 1.0; *fact = 1.0; *facn = 0.0;
    } else if (iter == 2) {
      *faco = 0.75; *fact = 0.25; *facn = *fact;
    } else {
      *faco = 1.0 / 3.0; *fact = 2.0 / 3.0; *facn = *fact;
    }
  } else if (type == 2) {
    if (iter == 1) {
      *faco = 1.0; *fact = 1.0; *facn = 0.0;
    } else {
      *faco = 0.5; *fact = 0.5; *facn = *fact;
    }
  } else {
    *faco = 1.0; *fact = 1.0; *facn = 0.0;
  }
}

// Stage arguments of one batched simulation: the same buffer roles as the
// single-grid driver (stage 1: U[0] -> U[1]; stage 2: U[1] -> U[2] (U[0]
// for rktype 2); stage 3: U[2] -> U[0]); primitive planes alternate.
__device__ __forceinline__ StageArgs batch_stage_args(SimDesc& S, int stage, int rk) {
  StageArgs a;
  rk_coefficients(stage, rk, &a.faco, &a.fact, &a.facn);
  a.stage = stage;
  a.nspc = 0;
  a.spcorg = nullptr;
  const int pin = (S.pcur + stage - 1) & 1;
  a.pin = S.P[pin];
  a.pout = S.P[pin ^ 1];
  a.uorg = S.U[0];
  if (stage == 1) {
    a.ucur = S.U[0];
    a.uout = S.U[1];
    a.phifac = S.phifac;
  } else if (stage == 2) {
    a.ucur = S.U[1];
    a.uout = rk == 2 ? S.U[0] : S.U[2];
    a.phifac = 1.0;
  } else {
    a.ucur = S.U[2];
    a.uout = S.U[0];
    a.phifac = 1.0;
  }
  a.gphi = nullptr;
  a.sc = &S.sc;
  a.plane = S.plane;
  a.gamma = S.gamma;
  a.gm1 = S.gm1;
  a.limiter = S.limiter;
  a.nvar = S.nvar;
  for (int d = 0; d < 3; d++) {
    a.tile[d] = 0;
    a.tiles[d] = S.tiles[d];
  }
  return a;
}

// tile kinds of the batched kernels: 0 = 3-D 8x8x8, 1 = 2-D xy 16x16,
// 2 = 1-D x 256
constexpr int kBatchKinds = 3;

// z slabs exchanging by push: a cell of the two bottom (top) layers also
// stores the primitive planes it just wrote into the low (high) neighbour's
// halo buffer, plane p layer l at (p * 2 + l) * nx * ny + i + nx * j, the
// layout the neighbour's staging reads.  On several GPUs the buffer is the
// neighbour's memory, so the exchange runs inside the stage, cell by cell.
__device__ __forceinline__ void push_boundary_layers(const GridDev& G, const StageArgs& A, const double* Po,
                                                     size_t c, int i, int j, int k) {
  const size_t hp = (size_t)G.n[0] * G.n[1], hc = (size_t)i + (size_t)G.n[0] * j, pl = A.plane;
  const int np = NP + A.nspc;
#pragma unroll
  for (int side = 0; side < 2; side++) {
    double* D = A.push[side];
    const int l = side == 0 ? k : k - (G.n[2] - 2);
    if (D == nullptr || l < 0 || l > 1) continue;
    const size_t o = (size_t)l * hp + hc;
    for (int p = 0; p < np; p++) D[(size_t)p * 2 * hp + o] = Po[(size_t)p * pl + c];
  }
}

// Spherical metric weights of the flux divergence of cell (i,j,k) along AX
// (rungekutta.f90:42-53 with metric.f90:105-125): the cell adds
// cw (fm F(low face) - fp F(high face)).  Along phi the reference has no face
// factor; fm = fp = 1 there, and multiplying by one is exact.
template <int AX>
__device__ __forceinline__ void sph_div_weights(const GridDev& G, int i, int j, int k, double& cw, double& fm,
                                                double& fp) {
  const SphGeo& M = G.sph;
  if constexpr (AX == 0) {  // idetg1, detg1 = xi1^2
    cw = M.idetg1[i + 2];
    fm = M.detg1[i + 1];
    fp = M.detg1[i + 2];
  } else if constexpr (AX == 1) {  // idetg2 = 1/(cos(j-1) - cos(j)) * sx1, detg2 = sin
    cw = M.ra2[j + 2] * M.sx1[i + 2];
    fm = M.sini[j + 1];
    fp = M.sini[j + 2];
  } else {  // idetg3 = idetg2 * dxi2 * idxi3 / fac_k (spherical), idxi3 (cylindrical)
    cw = M.crd == 1 ? G.g[2].idxi[k + 2]
                    : M.ra2[j + 2] * M.sx1[i + 2] * G.g[1].dxi[j + 2] * G.g[2].idxi[k + 2] / M.fac_k;
    fm = 1.0;
    fp = 1.0;
  }
}

// The gravitational potential at the neighbour o = -1 / +1 of cell c =
// (i,j,k) along axis a, with the ghost images the boundary pass of the
// hyperbolic solver forms: a periodic copy; on spherical grids copies at the
// inner radius and the poles and phi ~ 1/r beyond the outer radius
// (gravity_hyperbolic.f90:186-207, gbtype 1); on Cartesian grids the
// neighbouring z slab's layer or the Robin image phi ~ 1/r about the origin.
template <bool SPH>
__device__ __forceinline__ double gphi_at(const GridDev& G, const double* gphi, size_t c, int i, int j, int k,
                                          int a, int o) {
  int nb[3] = {i, j, k};
  nb[a] += o;
  if (nb[a] >= 0 && nb[a] < G.n[a]) return gphi[cidx(G, nb[0], nb[1], nb[2])];
  if (!SPH && a == 2 && G.ghalo[o > 0] != nullptr) return G.ghalo[o > 0][(size_t)i + (size_t)G.n[0] * j];
  if (G.bc[a][0][0] == 0) {
    nb[a] = nb[a] < 0 ? G.n[a] - 1 : 0;
    return gphi[cidx(G, nb[0], nb[1], nb[2])];
  }
  if constexpr (SPH) {
    if (a == 0 && o > 0) return gphi[c] * G.g[0].x[i + 2] / G.g[0].x[i + 3];
    return gphi[c];
  }
  const double xe = G.g[0].x[i + 2], ye = G.g[1].x[j + 2], ze = G.g[2].x[k + 2];
  const double xg = G.g[0].x[nb[0] + 2], yg = G.g[1].x[nb[1] + 2], zg = G.g[2].x[nb[2] + 2];
  const double re = sqrt(xe * xe + ye * ye + ze * ze), rg = sqrt(xg * xg + yg * yg + zg * zg);
  return gphi[c] * re / rg;
}

// -d(phi)/dx_a * rho of cell c along each axis (get_fieldforce,
// source.f90:177-228: centred differences on the non-uniform centres)
template <bool SPH>
__device__ __forceinline__ void gravity_force(const GridDev& G, const double* gphi, size_t c, int i, int j, int k,
                                              double d, double frc[3]) {
  const int ijk[3] = {i, j, k};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const AxisGeo& g = G.g[a];
    const int s = ijk[a];
    const double pm = gphi_at<SPH>(G, gphi, c, i, j, k, a, -1), p0 = gphi[c];
    const double pp = gphi_at<SPH>(G, gphi, c, i, j, k, a, 1);
    const double dxm = g.dx[s + 2], dxp = g.dx[s + 3], im = g.idx[s + 2], ip = g.idx[s + 3];
    frc[a] = -((dxm * ip * pp - dxp * im * pm) / (dxm + dxp) + (dxp - dxm) * im * ip * p0) * d;
  }
}

// Spherical geometric source terms (source.f90:113-143) of cell c, from the
// stage's input primitives with ptot = p + B^2/2 as `pressure` forms it
// (eos.f90:758-768), plus the gravity terms of :145-150 when grv is given,
// added to the flux divergence in acc[].
template <bool MAG>
__device__ __forceinline__ void sph_sources(const GridDev& G, const StageArgs& A, size_t c, int i, int j,
                                            double acc[9], const double* grv) {
  const SphGeo& M = G.sph;
  const size_t pl = A.plane;
  const double d = A.pin[c];
  const double v1 = A.pin[PV * pl + c], v2 = A.pin[(PV + 1) * pl + c], v3 = A.pin[(PV + 2) * pl + c];
  double pt = A.gm1 * A.pin[PEINT * pl + c];
  double b1 = 0.0, b2 = 0.0, b3 = 0.0;
  if (MAG) {
    b1 = A.pin[PB * pl + c];
    b2 = A.pin[(PB + 1) * pl + c];
    b3 = A.pin[(PB + 2) * pl + c];
    pt = pt + 0.5 * (b1 * b1 + b2 * b2 + b3 * b3);
  }
  if (M.crd == 1) {  // cylindrical (source.f90:88-111; phi unsolved, no gravity)
    const double s1 = M.sx1[i + 2];
    double r1 = (d * v2 * v2 + pt) * s1;
    double r2 = -(d * v1 * v2 * s1);
    if (MAG) {
      r1 = r1 - b2 * b2 * s1;
      r2 = r2 + b1 * b2 * s1;
      acc[6] = acc[6] + (b1 * v3 - b3 * v1) * s1;
    }
    acc[1] = acc[1] + r1;
    acc[2] = acc[2] + r2;
    return;
  }
  const double s1 = M.sx1[i + 2], sc = M.scot[j + 2];
  double r1 = (d * (v2 * v2 + v3 * v3) + 2.0 * pt) * s1;
  double r2 = G.solve[1] ? (-(d * v1 * v2) + (d * (v3 * v3) + pt) * sc) * s1 : 0.0;
  double r3 = (-(d * v1 * v3) - d * v2 * v3 * sc) * s1;
  if (MAG) {
    r1 = r1 - (b2 * b2 + b3 * b3) * s1;
    r2 = r2 + (b1 * b2 - b3 * b3 * sc) * s1;
    r3 = r3 + (b1 * b3 + b2 * b3 * sc) * s1;
    acc[6] = acc[6] + (b2 * v1 - b1 * v2) * s1;
    acc[7] = acc[7] + ((v2 * b3 - b2 * v3) * sc - (b1 * v3 - b3 * v1)) * s1;
  }
  if (grv != nullptr) {
    const double ss = M.sisin[j + 2];
    r1 = r1 + grv[0];
    r2 = r2 + grv[1] * s1;
    r3 = r3 + grv[2] * s1 * ss;
    acc[4] = acc[4] + (grv[0] * v1 + grv[1] * v2 * s1 + grv[2] * v3 * s1 * ss);
  }
  acc[1] = acc[1] + r1;
  acc[2] = acc[2] + r2;
  acc[3] = acc[3] + r3;
}

}  // namespace hmn
