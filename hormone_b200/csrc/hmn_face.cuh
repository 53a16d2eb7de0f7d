// hmn_face.cuh -- the limited slopes of one cell and the flux through one
// face in the reference's operation order, with every quotient formed by
// FastDiv (hmn_div.cuh) and an exact fallback; shared by the march
// (hmn_march.cu) and tile (hmn_kernels.cu) stages.  Results are bitwise
// those of IEEE division.
#pragma once
#include <cuda_runtime.h>

#include "hmn_div.cuh"
#include "hmn_math.cuh"
#include "hmn_tile.cuh"

namespace hmn {
namespace {

// Limited slopes of one cell along one axis from its two neighbours
// (interpolation.f90:49-163 with fluxlimiter.f90:40-75): pm, p0, pp point at
// staged quantity 0 of the cells, quantity q at [q * QS].  cg is the cell's
// global coordinate along the axis.  The same operations as axis_pass.
template <bool MAG, int LIM, int QS, class D>
__device__ __forceinline__ void slopes_with(const double* pm, const double* p0, const double* pp, const AxisGeo& g,
                                            int cg, double sl[NS], D& dv) {
  constexpr int nsl = MAG ? NS : S_B;
#pragma unroll
  for (int q = 0; q < NS; q++) sl[q] = 0.0;
  if constexpr (LIM == 0) {
    return;
  } else {
    constexpr int qmap[NS] = {Q_D, Q_E, Q_M + 0, Q_M + 1, Q_M + 2, Q_B + 0, Q_B + 1, Q_B + 2};
    const double hl = g.hl[cg + 2], hr = g.hr[cg + 2];
    double L[NS], R[NS];
    if constexpr (LIM == 1) {
      const double i0 = g.idx[cg + 2], i1 = g.idx[cg + 3], is = g.isum[cg + 2];
      const double ris = dv.rec(is);
#pragma unroll
      for (int q = 0; q < nsl; q++) {
        const double u0 = pm[qmap[q] * QS], u1 = p0[qmap[q] * QS], u2 = pp[qmap[q] * QS];
        const double du = lim_minmod(u0, u1, u2, i0, i1, is, dv, ris);
        sl[q] = du;
        L[q] = u1 - hl * du;
        R[q] = u1 + hr * du;
      }
    } else {
      const double cf = g.mcf[cg + 2], cb = g.mcb[cg + 2], ga = g.ga[cg + 2], gb = g.gb[cg + 2];
      const double rga = dv.rec(ga), rgb = dv.rec(gb);
#pragma unroll
      for (int q = 0; q < nsl; q++) {
        const double u0 = pm[qmap[q] * QS], u1 = p0[qmap[q] * QS], u2 = pp[qmap[q] * QS];
        const double du = lim_mmc(u0, u1, u2, cf, cb, ga, gb, dv, rga, rgb);
        sl[q] = du;
        L[q] = u1 - hl * du;
        R[q] = u1 + hr * du;
      }
    }
    double eintl = L[S_E] - dv.div(0.5 * (L[S_M] * L[S_M] + L[S_M + 1] * L[S_M + 1] + L[S_M + 2] * L[S_M + 2]),
                                   L[S_D], dv.rec(L[S_D]));
    double eintr = R[S_E] - dv.div(0.5 * (R[S_M] * R[S_M] + R[S_M + 1] * R[S_M + 1] + R[S_M + 2] * R[S_M + 2]),
                                   R[S_D], dv.rec(R[S_D]));
    if (MAG) {
      eintl = eintl - 0.5 * (L[S_B] * L[S_B] + L[S_B + 1] * L[S_B + 1] + L[S_B + 2] * L[S_B + 2]);
      eintr = eintr - 0.5 * (R[S_B] * R[S_B] + R[S_B + 1] * R[S_B + 1] + R[S_B + 2] * R[S_B + 2]);
    }
    const double em = pm[Q_EINT * QS], e0 = p0[Q_EINT * QS], ep = pp[Q_EINT * QS];
    if (eintl >= fmax2(em, e0) || eintl <= fmin2(em, e0) || eintr >= fmax2(e0, ep) || eintr <= fmin2(e0, ep)) {
#pragma unroll
      for (int q = 0; q < NS; q++) sl[q] = 0.0;
    }
  }
}

// The slopes with IEEE division, out of line: the rare path of slopes_of.
// Slope q goes to out[q * os].
template <bool MAG, int LIM, int QS>
__device__ __noinline__ void slopes_ieee(const double* pm, const double* p0, const double* pp, const AxisGeo* g,
                                         int cg, double* out, int os) {
  PlainDiv pd;
  double sl[NS];
  slopes_with<MAG, LIM, QS>(pm, p0, pp, *g, cg, sl, pd);
#pragma unroll
  for (int q = 0; q < NS; q++) out[q * os] = sl[q];
}

// The slopes with every quotient formed by FastDiv, recomputed with IEEE
// division where FastDiv could not vouch for one (bitwise the same result).
// One out-of-line copy serves every call site, so that warps in different
// phases of the march share instruction cache lines.  Slope q goes to
// out[q * os]: a caller that keeps slopes in shared memory passes its slot
// there, and nothing goes through the stack.
template <bool MAG, int LIM, int QS>
__device__ __noinline__ void slopes_fast(const double* pm, const double* p0, const double* pp, const AxisGeo* g,
                                         int cg, double* out, int os) {
  FastDiv fd;
  double sl[NS];
  slopes_with<MAG, LIM, QS>(pm, p0, pp, *g, cg, sl, fd);
  if (fd.bad) {
    slopes_ieee<MAG, LIM, QS>(pm, p0, pp, g, cg, out, os);
    return;
  }
#pragma unroll
  for (int q = 0; q < NS; q++) out[q * os] = sl[q];
}
template <bool MAG, int LIM, int QS>
__device__ __forceinline__ void slopes_of(const double* pm, const double* p0, const double* pp, const AxisGeo& g,
                                          int cg, double sl[NS]) {
  if constexpr (LIM == 0) {
#pragma unroll
    for (int q = 0; q < NS; q++) sl[q] = 0.0;
  } else {
    double tmp[NS];
    slopes_fast<MAG, LIM, QS>(pm, p0, pp, &g, cg, tmp, 1);
#pragma unroll
    for (int q = 0; q < NS; q++) sl[q] = tmp[q];
  }
}

// slopes_of written straight to out[q * os] (shared memory).
template <bool MAG, int LIM, int QS>
__device__ __forceinline__ void slopes_to(const double* pm, const double* p0, const double* pp, const AxisGeo& g,
                                          int cg, double* out, int os) {
  if constexpr (LIM == 0) {
#pragma unroll
    for (int q = 0; q < NS; q++) out[q * os] = 0.0;
  } else {
    slopes_fast<MAG, LIM, QS>(pm, p0, pp, &g, cg, out, os);
  }
}

// Flux through one face (numflux.f90:65-198 + hlldflux.f90): pl/pr give the
// staged quantities of the left and right cells, sl/sr their slopes (index
// functors), dx1 = xi - x(left), dx2 = x(right) - xi, (cn, c1, c2) the
// normal and tangential components.  fl[0..8] in the solver's order (mass,
// normal and tangential momenta, energy, normal B (phi flux), tangential B,
// ch^2 B_n).  Returns false (fl zero) where a face state has eint <= 0 or
// rho <= 0 (numflux.f90:117 -> error_flux).
template <bool MAG, class D, class PL, class PR, class SL, class SR>
__device__ __forceinline__ bool face_flux_with(PL pl, PR pr, SL sl, SR sr, double dx1, double dx2, int cn, int c1,
                                               int c2, double gamma, double gm1, double ch, double fl[9], D& dv) {
  const double dl = pl(Q_D) + dx1 * sl(S_D);
  const double dr = pr(Q_D) - dx2 * sr(S_D);
  const double el = pl(Q_E) + dx1 * sl(S_E);
  const double er = pr(Q_E) - dx2 * sr(S_E);
  const double rdl = dv.rec(dl), rdr = dv.rec(dr);
  const double v1l = dv.div(pl(Q_M + cn) + dx1 * sl(S_M + cn), dl, rdl);
  const double v1r = dv.div(pr(Q_M + cn) - dx2 * sr(S_M + cn), dr, rdr);
  const double v2l = dv.div(pl(Q_M + c1) + dx1 * sl(S_M + c1), dl, rdl);
  const double v2r = dv.div(pr(Q_M + c1) - dx2 * sr(S_M + c1), dr, rdr);
  const double v3l = dv.div(pl(Q_M + c2) + dx1 * sl(S_M + c2), dl, rdl);
  const double v3r = dv.div(pr(Q_M + c2) - dx2 * sr(S_M + c2), dr, rdr);
  double b1l = 0.0, b1r = 0.0, b2l = 0.0, b2r = 0.0, b3l = 0.0, b3r = 0.0, phil = 0.0, phir = 0.0;
  if (MAG) {
    b1l = pl(Q_B + cn) + dx1 * sl(S_B + cn);
    b1r = pr(Q_B + cn) - dx2 * sr(S_B + cn);
    b2l = pl(Q_B + c1) + dx1 * sl(S_B + c1);
    b2r = pr(Q_B + c1) - dx2 * sr(S_B + c1);
    b3l = pl(Q_B + c2) + dx1 * sl(S_B + c2);
    b3r = pr(Q_B + c2) - dx2 * sr(S_B + c2);
    // phi is never reconstructed: its slope is identically zero (allocations.f90)
    phil = pl(Q_PHI) + dx1 * 0.0;
    phir = pr(Q_PHI) - dx2 * 0.0;
  }
  const double eil = get_eint<MAG>(el, dl, v1l, v2l, v3l, b1l, b2l, b3l);
  const double eir = get_eint<MAG>(er, dr, v1r, v2r, v3r, b1r, b2r, b3r);
  if (eil <= 0.0 || dl <= 0.0 || eir <= 0.0 || dr <= 0.0) {
#pragma unroll
    for (int q = 0; q < 9; q++) fl[q] = 0.0;
    return false;
  }
  // eos_p_cs (eos.f90:209-219) with erad = 0
  const double ptl0 = gm1 * eil, ptr0 = gm1 * eir;
  const double csl = sqrt(dv.div(gamma * ptl0, dl, rdl)), csr = sqrt(dv.div(gamma * ptr0, dr, rdr));
  const double ptl = ptl0 + 0.5 * (b1l * b1l + b2l * b2l + b3l * b3l);
  const double ptr = ptr0 + 0.5 * (b1r * b1r + b2r * b2r + b3r * b3r);
  const double cfl = get_cf(dl, csl, b1l, b2l, b3l, dv, rdl);
  const double cfr = get_cf(dr, csr, b1r, b2r, b3r, dv, rdr);
  hlld(fl, cfl, cfr, v1l, v1r, v2l, v2r, v3l, v3r, dl, dr, el, er, ptl, ptr, b1l, b1r, b2l, b2r, b3l, b3r, phil, phir,
       ch, dv);
  return true;
}

// Store a face flux: with os == 0, fl in the solver's order to out[0..8];
// otherwise rotated back into the conserved slots (numflux.f90:186-198,
// 359-371, 531-543), slot v to out[v * os].
__device__ __forceinline__ void put_flux(const double fl[9], int cn, int c1, int c2, double* out, int os) {
  if (os == 0) {
#pragma unroll
    for (int q = 0; q < 9; q++) out[q] = fl[q];
    return;
  }
  out[ICNT * os] = fl[0];
  out[(IMO1 + cn) * os] = fl[1];
  out[(IMO1 + c1) * os] = fl[2];
  out[(IMO1 + c2) * os] = fl[3];
  out[IENE * os] = fl[4];
  out[(IMG1 + cn) * os] = fl[5];
  out[(IMG1 + c1) * os] = fl[6];
  out[(IMG1 + c2) * os] = fl[7];
  out[I9WV * os] = fl[8];
}

// The face flux with IEEE division, out of line: the rare path of
// face_flux.  pl/pr: staged quantity 0 of the cells (stride QS); sl/sr:
// slope 0 (strides ssl, ssr); out/os as put_flux.
template <bool MAG, int QS>
__device__ __noinline__ bool face_flux_ieee(const double* pl, const double* pr, const double* sl, int ssl,
                                            const double* sr, int ssr, double dx1, double dx2, int cn, int c1, int c2,
                                            double gamma, double gm1, double ch, double* out, int os) {
  PlainDiv pd;
  double fl[9];
  const bool ok = face_flux_with<MAG>([&](int q) { return pl[q * QS]; }, [&](int q) { return pr[q * QS]; },
                                      [&](int q) { return sl[q * ssl]; }, [&](int q) { return sr[q * ssr]; }, dx1,
                                      dx2, cn, c1, c2, gamma, gm1, ch, fl, pd);
  put_flux(fl, cn, c1, c2, out, os);
  return ok;
}

// The face flux with every quotient formed by FastDiv, recomputed with IEEE
// division where FastDiv could not vouch for one (bitwise the same result);
// one out-of-line copy for the x, y and z faces.  Arguments as
// face_flux_ieee.  A caller that keeps fluxes in shared memory passes its
// slot and stride, and nothing goes through the stack.
template <bool MAG, int QS>
__device__ __noinline__ bool face_flux_fast(const double* pl, const double* pr, const double* sl, int ssl,
                                            const double* sr, int ssr, double dx1, double dx2, int cn, int c1, int c2,
                                            double gamma, double gm1, double ch, double* out, int os) {
  FastDiv fd;
  double fl[9];
  const bool ok = face_flux_with<MAG>([&](int q) { return pl[q * QS]; }, [&](int q) { return pr[q * QS]; },
                                      [&](int q) { return sl[q * ssl]; }, [&](int q) { return sr[q * ssr]; }, dx1,
                                      dx2, cn, c1, c2, gamma, gm1, ch, fl, fd);
  if (fd.bad)
    return face_flux_ieee<MAG, QS>(pl, pr, sl, ssl, sr, ssr, dx1, dx2, cn, c1, c2, gamma, gm1, ch, out, os);
  put_flux(fl, cn, c1, c2, out, os);
  return ok;
}

}  // namespace
}  // namespace hmn
