// hmn_math.cuh -- per-cell and per-face arithmetic of HORMONE's explicit step,
// in the operation order of the Fortran reference (every product, sum and
// quotient below is one IEEE binary64 operation; the including translation
// unit is compiled with --fmad=false so nothing is fused).
//
// Reference routines (paths in the HORMONE tree):
//   minmod / modified_mc   src/main/fluxlimiter.f90:40-56, 58-75
//   get_eint               src/main/eos.f90:846-866
//   get_cf                 src/main/eos.f90:351-365
//   eos_p_cs (ideal gas)   src/main/eos.f90:195-242
//   hlldflux + fstar       src/main/hlldflux.f90:19-179
#pragma once
#include <cuda_runtime.h>

namespace hmn {

// Fortran SIGN(a,b): |a| with the sign bit of b (honours -0).
template <typename T>
__device__ __forceinline__ T fsign(T a, T b) { return copysign(fabs(a), b); }
// MIN/MAX in the argument order the reference evaluates them.
template <typename T>
__device__ __forceinline__ T fmin2(T a, T b) { return a < b ? a : b; }
template <typename T>
__device__ __forceinline__ T fmax2(T a, T b) { return a > b ? a : b; }

// Division policies: div(a, b, r) is a/b, where r = rec(b) was formed once
// for every quotient with the denominator b.  PlainDiv divides (r is b
// itself); FastDiv (hmn_div.cuh) forms RN(1/b) once and corrects each
// quotient to RN(a/b), flagging operands it cannot take.
struct PlainDiv {
  template <typename T>
  __device__ __forceinline__ T rec(T b) { return b; }
  template <typename T>
  __device__ __forceinline__ T div(T a, T b, T) { return a / b; }
};

// Generalised minmod with theta = 1.4 on inverse spacings (fluxlimiter.f90:40-56).
// i0 = 1/dx(c), i1 = 1/dx(c+1), isum = i0 + i1; risum = dv.rec(isum).
template <class D>
__device__ __forceinline__ double lim_minmod(double u0, double u1, double u2, double i0, double i1, double isum,
                                             D& dv, double risum) {
  double x = 1.4 * (u2 - u1) * i1;
  double y = 1.4 * (u1 - u0) * i0;
  double z = dv.div((u2 - u0) * i0 * i1, isum, risum);
  double s = fsign(1.0, x);
  double m = fabs(x);
  m = fmin2(m, s * y);
  m = fmin2(m, s * z);
  return s * fmax2(0.0, m);
}
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

// Modified MC (fluxlimiter.f90:58-75).  Grid factors precomputed per cell:
// cf = (x(c+1)-x(c))/(xi(c)-x(c)), cb = (x(c)-x(c-1))/(x(c)-xi(c-1)),
// ga = x(c+1)-x(c), gb = x(c)-x(c-1).
// With a division policy: rga = dv.rec(ga), rgb = dv.rec(gb).
template <class D>
__device__ __forceinline__ double lim_mmc(double u0, double u1, double u2, double cf, double cb, double ga, double gb,
                                          D& dv, double rga, double rgb) {
  double top = dv.div((u1 - u0) * ga, gb, rgb);
  double bot = u2 - u1;
  double sig = fsign(1.0, bot);
  double m = sig * 0.5 * (bot + top);
  m = fmin2(m, sig * cf * bot);
  m = fmin2(m, sig * cb * top);
  return dv.div(sig * fmax2(0.0, m), ga, rga);
}
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

// Fast magnetosonic speed along b1 (eos.f90:351-365); rd = dv.rec(d).
template <typename T, class D>
__device__ __forceinline__ T get_cf(T d, T cs, T b1, T b2, T b3, D& dv, T rd) {
  T asq = cs * cs;
  T bb1 = dv.div(b1 * b1, d, rd);
  T bb2 = dv.div(b2 * b2, d, rd);
  T bb3 = dv.div(b3 * b3, d, rd);
  T bbsq = bb1 + bb2 + bb3;
  T t = asq + bbsq;
  return sqrt(T(0.5) * (t + sqrt(t * t - T(4.0) * asq * bb1)));
}
template <typename T>
__device__ __forceinline__ T get_cf(T d, T cs, T b1, T b2, T b3) {
  T asq = cs * cs;
  T bb1 = b1 * b1 / d;
  T bb2 = b2 * b2 / d;
  T bb3 = b3 * b3 / d;
  T bbsq = bb1 + bb2 + bb3;
  T t = asq + bbsq;
  return sqrt(T(0.5) * (t + sqrt(t * t - T(4.0) * asq * bb1)));
}

// Face flux of one interface: HLLD (Miyoshi & Kusano 2005) with the GLM mixing
// of the normal field and phi (hlldflux.f90:19-150), then the flux of the
// selected state (fstar, hlldflux.f90:156-179).  f[0..8] = mass, normal and
// two tangential momenta, energy, phi-flux (normal B), two tangential B,
// ch^2*B_n.  T = double in the FP64 path; the mixed-precision path
// instantiates it for float.
template <typename T, class D>
__device__ __forceinline__ void hlld(T f[9], T cfl, T cfr, T v1l, T v1r, T v2l, T v2r, T v3l, T v3r, T dl, T dr, T el,
                                     T er, T ptl, T ptr, T b1l, T b1r, T b2l, T b2r, T b3l, T b3r, T phil, T phir,
                                     T ch, D& dvp) {
  const T h = T(0.5), one = T(1.0), zero = T(0.0);
  const T b1 = h * ((b1l + b1r) - dvp.div(phir - phil, ch, dvp.rec(ch)));
  const T phi = h * ((phil + phir) - (b1r - b1l) * ch);
  const T sl = fmin2(fmin2(v1r - cfr, v1l - cfl), zero);
  const T sr = fmax2(fmax2(v1r + cfr, v1l + cfl), zero);
  const T wl = sl - v1l, wr = sr - v1r;  // S - v on each side
  const T den = wr * dr - wl * dl;
  const T rden = dvp.rec(den);
  const T sm = dvp.div(wr * dr * v1r - wl * dl * v1l - ptr + ptl, den, rden);
  const T slsm = sl - sm, srsm = sr - sm;
  const T rslsm = dvp.rec(slsm), rsrsm = dvp.rec(srsm);
  const T dla0 = dvp.div(dl * wl, slsm, rslsm);
  const T dra0 = dvp.div(dr * wr, srsm, rsrsm);
  const T sqla = sqrt(dla0), sqra = sqrt(dra0);
  const T sla = sm - dvp.div(fabs(b1), sqla, dvp.rec(sqla));
  const T sra = sm + dvp.div(fabs(b1), sqra, dvp.rec(sqra));
  const T pta = dvp.div(wr * dr * ptl - wl * dl * ptr + dl * dr * wr * wl * (v1r - v1l), den, rden);
  const T b1b1 = b1 * b1;
  const T denl = dl * wl * (sl - sm) - b1b1;
  const T denr = dr * wr * (sr - sm) - b1b1;
  const T rdenl = dvp.rec(denl), rdenr = dvp.rec(denr);
  const T v2la = v2l - dvp.div(b1 * b2l * (sm - v1l), denl, rdenl);
  const T v2ra = v2r - dvp.div(b1 * b2r * (sm - v1r), denr, rdenr);
  const T v3la = v3l - dvp.div(b1 * b3l * (sm - v1l), denl, rdenl);
  const T v3ra = v3r - dvp.div(b1 * b3r * (sm - v1r), denr, rdenr);
  const T numl = dl * wl * wl - b1b1;
  const T numr = dr * wr * wr - b1b1;
  const T b2la = dvp.div(b2l * numl, denl, rdenl);
  const T b2ra = dvp.div(b2r * numr, denr, rdenr);
  const T b3la = dvp.div(b3l * numl, denl, rdenl);
  const T b3ra = dvp.div(b3r * numr, denr, rdenr);
  const T ela = dvp.div(wl * el - ptl * v1l + pta * sm +
                           b1 * ((v1l * b1 + v2l * b2l + v3l * b3l) - (sm * b1 + v2la * b2la + v3la * b3la)),
                       slsm, rslsm);
  const T era = dvp.div(wr * er - ptr * v1r + pta * sm +
                           b1 * ((v1r * b1 + v2r * b2r + v3r * b3r) - (sm * b1 + v2ra * b2ra + v3ra * b3ra)),
                       srsm, rsrsm);
  const T s1 = fsign(one, b1);
  const T sqsum = sqla + sqra;
  const T rsqsum = dvp.rec(sqsum);
  const T v2aa = dvp.div(sqla * v2la + sqra * v2ra + (b2ra - b2la) * s1, sqsum, rsqsum);
  const T v3aa = dvp.div(sqla * v3la + sqra * v3ra + (b3ra - b3la) * s1, sqsum, rsqsum);
  const T sqlr = sqrt(dla0 * dra0);
  const T b2aa = dvp.div(sqla * b2ra + sqra * b2la + sqlr * (v2ra - v2la) * s1, sqsum, rsqsum);
  const T b3aa = dvp.div(sqla * b3ra + sqra * b3la + sqlr * (v3ra - v3la) * s1, sqsum, rsqsum);
  const T vbaa = v2aa * b2aa + v3aa * b3aa;
  const T eraa = era + s1 * sqra * ((v2ra * b2ra + v3ra * b3ra) - vbaa);
  const T elaa = ela - s1 * sqla * ((v2la * b2la + v3la * b3la) - vbaa);
  // branch-free selection of the state at x/t = 0 (hlldflux.f90:113-145)
  const T signsm = fsign(h, sm);
  const T wsla = h + fsign(h, sla);
  const T wsra = h + fsign(h, -sra);
  const T wslr = h - fsign(h, sla * sra);
  const T d = (h + signsm) * dla0 + (h - signsm) * dra0;
  const T v2 = wsla * v2la + wslr * v2aa + wsra * v2ra;
  const T v3 = wsla * v3la + wslr * v3aa + wsra * v3ra;
  const T bb2 = wsla * b2la + wslr * b2aa + wsra * b2ra;
  const T bb3 = wsla * b3la + wslr * b3aa + wsra * b3ra;
  const T e = wsla * ela + (h - fsign(h, sla * sm)) * elaa + (h + fsign(h, -(sm * sra))) * eraa +
                   (h - fsign(h, sra)) * era;
  const T v1 = sm, p = pta;
  const T dv = d * v1;
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

// The same with plain division (every caller without a division policy).
template <typename T>
__device__ __forceinline__ void hlld(T f[9], T cfl, T cfr, T v1l, T v1r, T v2l, T v2r, T v3l, T v3r, T dl, T dr, T el,
                                     T er, T ptl, T ptr, T b1l, T b1r, T b2l, T b2r, T b3l, T b3r, T phil, T phir,
                                     T ch) {
  PlainDiv dv;
  hlld(f, cfl, cfr, v1l, v1r, v2l, v2r, v3l, v3r, dl, dr, el, er, ptl, ptr, b1l, b1r, b2l, b2r, b3l, b3r, phil, phir, ch,
       dv);
}

}  // namespace hmn
