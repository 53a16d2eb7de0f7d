// hmn_math.cuh -- per-cell and per-face arithmetic of HORMONE's explicit step,
// in the operation order of the Fortran reference (every product, sum and
// quotient below is one IEEE binary64 operation; the including translation
// unit is compiled with --fmad=false so nothing is fused).
//
// Reference routines (paths in the HORMONE tree):
//   minmod / modified_mc   src/main/fluxlimiter.f90:94-129
//   get_eint               src/main/eos.f90:846-866
//   get_cf                 src/main/eos.f90:351-365
//   eos_p_cs (ideal gas)   src/main/eos.f90:195-242
//   hlldflux + fstar       src/main/hlldflux.f90:19-179
#pragma once
#include <cuda_runtime.h>

namespace hmn {

// Fortran SIGN(a,b): |a| with the sign bit of b (honours -0).
__device__ __forceinline__ double fsign(double a, double b) { return copysign(fabs(a), b); }
// MIN/MAX in the argument order the reference evaluates them.
__device__ __forceinline__ double fmin2(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double fmax2(double a, double b) { return a > b ? a : b; }

// Generalised minmod with theta = 1.4 on inverse spacings (fluxlimiter.f90:94-110).
// i0 = 1/dx(c), i1 = 1/dx(c+1), isum = i0 + i1.
__device__ __forceinline__ double lim_minmod(double u0, double u1, double u2, double i0, double i1, double isum) {
  double x = 1.4 * (u2 - u1) * i1;
  double y = 1.4 * (u1 - u0) * i0;
  double z = (u2 - u0) * i0 * i1 / isum;
  double s = fsign(1.0, x);
  double m = fabs(x);
  m = fmin2(m, s * y);
  m = fmin2(m, s * z);
  return s * fmax2(0.0, m);
}

// Modified MC (fluxlimiter.f90:112-129).  Grid factors precomputed per cell:
// cf = (x(c+1)-x(c))/(xi(c)-x(c)), cb = (x(c)-x(c-1))/(x(c)-xi(c-1)),
// ga = x(c+1)-x(c), gb = x(c)-x(c-1).
__device__ __forceinline__ double lim_mmc(double u0, double u1, double u2, double cf, double cb, double ga,
                                          double gb) {
  double top = (u1 - u0) * ga / gb;
  double bot = u2 - u1;
  double sig = fsign(1.0, bot);
  double m = sig * 0.5 * (bot + top);
  m = fmin2(m, sig * cf * bot);
  m = fmin2(m, sig * cb * top);
  return sig * fmax2(0.0, m) / ga;
}

// Internal energy from total energy (eos.f90:846-866).
template <bool MAG>
__device__ __forceinline__ double get_eint(double etot, double d, double v1, double v2, double v3, double b1,
                                           double b2, double b3) {
  double vsq = v1 * v1 + v2 * v2 + v3 * v3;
  double ei = etot - 0.5 * d * vsq;
  if (MAG) {
    double bsq = b1 * b1 + b2 * b2 + b3 * b3;
    ei = ei - 0.5 * bsq;
  }
  return ei;
}

// Fast magnetosonic speed along b1 (eos.f90:351-365).
__device__ __forceinline__ double get_cf(double d, double cs, double b1, double b2, double b3) {
  double asq = cs * cs;
  double bb1 = b1 * b1 / d;
  double bb2 = b2 * b2 / d;
  double bb3 = b3 * b3 / d;
  double bbsq = bb1 + bb2 + bb3;
  double t = asq + bbsq;
  return sqrt(0.5 * (t + sqrt(t * t - 4.0 * asq * bb1)));
}

// Face flux of one interface: HLLD (Miyoshi & Kusano 2005) with the GLM mixing
// of the normal field and phi (hlldflux.f90:19-150), then the flux of the
// selected state (fstar, hlldflux.f90:156-179).  f[0..8] = mass, normal and
// two tangential momenta, energy, phi-flux (normal B), two tangential B,
// ch^2*B_n.
__device__ __forceinline__ void hlld(double f[9], double cfl, double cfr, double v1l, double v1r, double v2l,
                                     double v2r, double v3l, double v3r, double dl, double dr, double el, double er,
                                     double ptl, double ptr, double b1l, double b1r, double b2l, double b2r,
                                     double b3l, double b3r, double phil, double phir, double ch) {
  const double b1 = 0.5 * ((b1l + b1r) - (phir - phil) / ch);
  const double phi = 0.5 * ((phil + phir) - (b1r - b1l) * ch);
  const double sl = fmin2(fmin2(v1r - cfr, v1l - cfl), 0.0);
  const double sr = fmax2(fmax2(v1r + cfr, v1l + cfl), 0.0);
  const double wl = sl - v1l, wr = sr - v1r;  // S - v on each side
  const double den = wr * dr - wl * dl;
  const double sm = (wr * dr * v1r - wl * dl * v1l - ptr + ptl) / den;
  const double dla0 = dl * wl / (sl - sm);
  const double dra0 = dr * wr / (sr - sm);
  const double sqla = sqrt(dla0), sqra = sqrt(dra0);
  const double sla = sm - fabs(b1) / sqla;
  const double sra = sm + fabs(b1) / sqra;
  const double pta = (wr * dr * ptl - wl * dl * ptr + dl * dr * wr * wl * (v1r - v1l)) / den;
  const double b1b1 = b1 * b1;
  const double denl = dl * wl * (sl - sm) - b1b1;
  const double denr = dr * wr * (sr - sm) - b1b1;
  const double v2la = v2l - b1 * b2l * (sm - v1l) / denl;
  const double v2ra = v2r - b1 * b2r * (sm - v1r) / denr;
  const double v3la = v3l - b1 * b3l * (sm - v1l) / denl;
  const double v3ra = v3r - b1 * b3r * (sm - v1r) / denr;
  const double numl = dl * wl * wl - b1b1;
  const double numr = dr * wr * wr - b1b1;
  const double b2la = b2l * numl / denl;
  const double b2ra = b2r * numr / denr;
  const double b3la = b3l * numl / denl;
  const double b3ra = b3r * numr / denr;
  const double ela = (wl * el - ptl * v1l + pta * sm +
                      b1 * ((v1l * b1 + v2l * b2l + v3l * b3l) - (sm * b1 + v2la * b2la + v3la * b3la))) /
                     (sl - sm);
  const double era = (wr * er - ptr * v1r + pta * sm +
                      b1 * ((v1r * b1 + v2r * b2r + v3r * b3r) - (sm * b1 + v2ra * b2ra + v3ra * b3ra))) /
                     (sr - sm);
  const double s1 = fsign(1.0, b1);
  const double sqsum = sqla + sqra;
  const double v2aa = (sqla * v2la + sqra * v2ra + (b2ra - b2la) * s1) / sqsum;
  const double v3aa = (sqla * v3la + sqra * v3ra + (b3ra - b3la) * s1) / sqsum;
  const double sqlr = sqrt(dla0 * dra0);
  const double b2aa = (sqla * b2ra + sqra * b2la + sqlr * (v2ra - v2la) * s1) / sqsum;
  const double b3aa = (sqla * b3ra + sqra * b3la + sqlr * (v3ra - v3la) * s1) / sqsum;
  const double vbaa = v2aa * b2aa + v3aa * b3aa;
  const double eraa = era + s1 * sqra * ((v2ra * b2ra + v3ra * b3ra) - vbaa);
  const double elaa = ela - s1 * sqla * ((v2la * b2la + v3la * b3la) - vbaa);
  // branch-free selection of the state at x/t = 0 (hlldflux.f90:113-145)
  const double signsm = fsign(0.5, sm);
  const double wsla = 0.5 + fsign(0.5, sla);
  const double wsra = 0.5 + fsign(0.5, -sra);
  const double wslr = 0.5 - fsign(0.5, sla * sra);
  const double d = (0.5 + signsm) * dla0 + (0.5 - signsm) * dra0;
  const double v2 = wsla * v2la + wslr * v2aa + wsra * v2ra;
  const double v3 = wsla * v3la + wslr * v3aa + wsra * v3ra;
  const double bb2 = wsla * b2la + wslr * b2aa + wsra * b2ra;
  const double bb3 = wsla * b3la + wslr * b3aa + wsra * b3ra;
  const double e = wsla * ela + (0.5 - fsign(0.5, sla * sm)) * elaa + (0.5 + fsign(0.5, -(sm * sra))) * eraa +
                   (0.5 - fsign(0.5, sra)) * era;
  const double v1 = sm, p = pta;
  const double dv = d * v1;
  f[0] = dv;
  f[1] = dv * v1 + p - b1 * b1;
  f[2] = dv * v2 - b1 * bb2;
  f[3] = dv * v3 - b1 * bb3;
  f[4] = (e + p) * v1 - b1 * (v1 * b1 + v2 * bb2 + v3 * bb3);
  f[5] = phi;
  f[6] = bb2 * v1 - b1 * v2;
  f[7] = bb3 * v1 - b1 * v3;
  f[8] = ch * ch * b1;
}

}  // namespace hmn
