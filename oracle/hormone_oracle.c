/*
 * hormone_oracle.c -- CPU restatement of HORMONE's explicit FP64 MHD step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference legs may load it.  The product (hormone_b200/) never links,
 * imports or calls it.
 *
 * It restates, pass by pass and with the reference's floating-point operation
 * order, the Fortran routines listed below (paths relative to the HORMONE
 * source tree).  The reference cannot be compiled in this environment (it is
 * Fortran 90 and no Fortran compiler exists), so this restatement is pinned
 * instead against the reference's own golden binaries
 * tests/{sodshock,briowushock}_{x,y,z}[_flat].bin and
 * tests/orszagtang_{xy,yz,xz}[_flat].bin with the norms of
 * src/main/tests.f90:46-292.
 *
 *   grid            src/main/gridset.f90:40-80 (uniform Cartesian),
 *                   :294-423 (spherical polar r, theta, phi), :145-292
 *                   (cylindrical R, phi, z without a solved phi)
 *   metric          src/main/metric.f90:26-51 (Cartesian), :53-100
 *                   (cylindrical), :102-151 (spherical)
 *   limiters        src/main/fluxlimiter.f90:40-56 (minmod), 58-75 (modified_mc)
 *   slopes          src/main/interpolation.f90:49-484
 *   face fluxes     src/main/numflux.f90:46-563
 *   HLLD + GLM      src/main/hlldflux.f90:19-179
 *   EOS (ideal)     src/main/eos.f90:195-274,351-365,742-866
 *   source          src/main/source.f90:14-85,177-228; cylindrical geometric
 *                   terms :88-111; spherical :113-150, pinned by
 *                   tests/sedov_default[_flat].bin
 *   RK + primitive  src/main/rungekutta.f90:16-232
 *   boundaries      src/main/boundarycondition.f90:14-1442 (codes 0-3; 4/5
 *                   linear extrapolation as :302-327,419-468; 9 Dirichlet
 *                   as :104-115,196-212 from per-face ghost values; 10 at
 *                   the inner x3 face: ghosts never rewritten, the face
 *                   flux from fluxboundary.f90:42-87)
 *   timestep        src/main/timestep.f90:15-183
 *   phidamp         src/main/source.f90:239-260
 *   hyperbolic grav src/main/gravity_hyperbolic.f90:19-125,230-280 with a
 *                   Cartesian Laplacian (the reference has no Cartesian form;
 *                   parity of that part is unpinned)
 *   passive scalars src/main/interpolation.f90:126-145 (slopes),
 *                   src/main/numflux.f90:200-212 (upwinded, renormalised
 *                   fluxes), src/main/rungekutta.f90:61-86 (update),
 *                   src/main/boundarycondition.f90 (scalar images),
 *                   pinned by tests/KHinstability[_flat].bin
 *   step order      src/main/hormone.f90:124-179, src/main/hydro.f90:15-52
 *
 * Build with -ffp-contract=off: every + - * / sqrt is a single IEEE binary64
 * operation, as in the reference built without optimisation.
 */
#include <math.h>
#include <quadmath.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define HMO_OK 0
#define HMO_ENEG_EINT -2 /* negative internal energy (numflux.f90:579, eos.f90:833) */
#define HMO_EBADCFG -4

enum { ICNT = 0, IMO1 = 1, IMO2 = 2, IMO3 = 3, IENE = 4, IMG1 = 5, IMG2 = 6, IMG3 = 7, I9WV = 8 };
enum { S_D = 0, S_E, S_M1, S_M2, S_M3, S_B1, S_B2, S_B3, NSLOPE };
#define MAXSPC 8

typedef struct {
  int n[3];           /* interior cells per axis */
  int solve[3], dim, mag_on, glm, nvar;
  int bc[3][2][2];    /* [axis][0 inner,1 outer][0 scalar,1 vector] */
  int limiter;        /* 0 flat, 1 minmod, 2 modified_mc */
  int rktype;
  int outstyle, endstyle;
  double gamma, courant, alpha9wave;
  /* hyperbolic gravity */
  int gravswitch, grktype, maxtngrv;
  double HGfac, hgcfl, alphagrv, G;
  /* grid arrays per axis, offset +2, length n+4 */
  double *x[3], *xi[3], *dx[3], *dxi[3], *idx[3], *idxi[3];
  size_t sx, sy, ncell; /* ghosted strides */
  /* ghosted primitive arrays */
  double *d, *p, *e, *v[3], *b[3], *phi, *eint, *cs, *ptot;
  double *u[9], *uorg[9], *flux[3][9], *src[9];
  double *slope[3][NSLOPE], *dphi;
  double *grvphi, *grvpsi, *gorg1, *gorg2, *lapphi, *hgsrc, *gsrc, *grv[3];
  /* passive scalars (compswitch 2): mass fractions, ghosted */
  int spn;
  double *spc[MAXSPC], *spcorg[MAXSPC], *dspc[3][MAXSPC], *spcflx[3][MAXSPC];
  /* Dirichlet ghost values per face: 8 + spn planes (d, p, v1..3, b1..3,
     spc) x 2 layers x face cells, layer l at coordinate -2+l (inner) or n+l */
  double *dir[3][2];
  /* boundary code 10 at the inner x3 face: the flux through that face,
     9 + spn values in conserved order (fluxboundary.f90:42-87) */
  double *fbflux;
  /* coordinate system: 0 Cartesian, 2 spherical polar (r, theta, phi) with
     the metric factors of metric.f90:102-151 (offset +2 like the axes) */
  int crdnt;
  double *detg1, *idetg1, *sx1;   /* r faces / cells */
  double *sini, *cosi, *scot;     /* theta faces / cells */
  double *sinc, *sisin;           /* sin of the arithmetic theta centres; dtheta/(cos-cos) */
  double xi1s;                    /* inner radius (the inner-boundary term of the gravity coefficients) */
  double fac_j, fac_k;
  /* scalars */
  double dt, ch, time, t_out, t_end, dt_out, cfmax;
  double cgrav, cgrav_old, dtgrav, dtg_unit, grvtime;
  int tn, tnlim, rungen;
  int err, err_i, err_j, err_k;
} Oracle;

#define IX(o, i, j, k) ((size_t)((i) + 2) + (o)->sx * ((size_t)((j) + 2) + (o)->sy * (size_t)((k) + 2)))

static inline double fsign(double a, double b) { return copysign(fabs(a), b); } /* Fortran SIGN */
static inline double fmin2(double a, double b) { return a < b ? a : b; }
static inline double fmax2(double a, double b) { return a > b ? a : b; }

static double *zalloc(size_t n) {
  double *p = (double *)calloc(n ? n : 1, sizeof(double));
  return p;
}

/* ------------------------------------------------------------------------ */
/* creation                                                                   */

Oracle *hmo_create(int nx, int ny, int nz, int mag_on, int limiter, int rktype, double gamma, double courant,
                   double alpha9wave, const int *bc /* 12 ints [axis][io][sv] */) {
  Oracle *o = (Oracle *)calloc(1, sizeof(Oracle));
  o->n[0] = nx; o->n[1] = ny; o->n[2] = nz;
  /* checksetup.f90:42-75 */
  o->dim = 0;
  for (int a = 0; a < 3; a++) { o->solve[a] = o->n[a] > 1; o->dim += o->solve[a]; }
  o->mag_on = mag_on;
  o->glm = mag_on && o->dim > 1;
  o->nvar = 5 + (mag_on ? 3 : 0) + (o->glm ? 1 : 0);
  memcpy(o->bc, bc, sizeof(o->bc));
  /* checksetup.f90:118-128: unsolved directions get outgoing/free codes */
  if (!o->solve[0]) for (int io = 0; io < 2; io++) for (int sv = 0; sv < 2; sv++) o->bc[0][io][sv] = 2;
  if (!o->solve[1]) for (int io = 0; io < 2; io++) for (int sv = 0; sv < 2; sv++) o->bc[1][io][sv] = 3;
  if (!o->solve[2]) for (int io = 0; io < 2; io++) for (int sv = 0; sv < 2; sv++) o->bc[2][io][sv] = 3;
  o->limiter = limiter; o->rktype = rktype;
  o->gamma = gamma; o->courant = courant; o->alpha9wave = alpha9wave;
  o->outstyle = 1; o->endstyle = 1;
  o->sx = (size_t)nx + 4; o->sy = (size_t)ny + 4;
  o->ncell = o->sx * o->sy * ((size_t)nz + 4);
  size_t N = o->ncell;
  for (int a = 0; a < 3; a++) {
    size_t L = (size_t)o->n[a] + 4;
    o->x[a] = zalloc(L); o->xi[a] = zalloc(L); o->dx[a] = zalloc(L);
    o->dxi[a] = zalloc(L); o->idx[a] = zalloc(L); o->idxi[a] = zalloc(L);
  }
  o->d = zalloc(N); o->p = zalloc(N); o->e = zalloc(N); o->phi = zalloc(N);
  o->eint = zalloc(N); o->cs = zalloc(N); o->ptot = zalloc(N); o->dphi = zalloc(N);
  for (int a = 0; a < 3; a++) { o->v[a] = zalloc(N); o->b[a] = zalloc(N); o->grv[a] = zalloc(N); }
  for (int q = 0; q < 9; q++) {
    o->u[q] = zalloc(N); o->uorg[q] = zalloc(N); o->src[q] = zalloc(N);
    for (int a = 0; a < 3; a++) o->flux[a][q] = zalloc(N);
  }
  for (int a = 0; a < 3; a++) for (int s = 0; s < NSLOPE; s++) o->slope[a][s] = zalloc(N);
  /* allocations.f90: strictly positive quantities start at 1 */
  for (size_t c = 0; c < N; c++) { o->d[c] = 1.0; o->p[c] = 1.0; o->e[c] = 1.0; o->eint[c] = 1.0; o->cs[c] = 1.0; o->ptot[c] = 1.0; }
  o->grvphi = zalloc(N); o->grvpsi = zalloc(N); o->gorg1 = zalloc(N); o->gorg2 = zalloc(N);
  o->lapphi = zalloc(N); o->hgsrc = zalloc(N); o->gsrc = zalloc(N);
  o->detg1 = zalloc((size_t)nx + 4); o->idetg1 = zalloc((size_t)nx + 4); o->sx1 = zalloc((size_t)nx + 4);
  o->sini = zalloc((size_t)ny + 4); o->cosi = zalloc((size_t)ny + 4); o->scot = zalloc((size_t)ny + 4);
  o->sinc = zalloc((size_t)ny + 4); o->sisin = zalloc((size_t)ny + 4);
  o->fac_j = 1.0; o->fac_k = 1.0;
  return o;
}

void hmo_destroy(Oracle *o) {
  if (!o) return;
  for (int a = 0; a < 3; a++) {
    free(o->x[a]); free(o->xi[a]); free(o->dx[a]); free(o->dxi[a]); free(o->idx[a]); free(o->idxi[a]);
    free(o->v[a]); free(o->b[a]); free(o->grv[a]);
    for (int s = 0; s < NSLOPE; s++) free(o->slope[a][s]);
  }
  free(o->d); free(o->p); free(o->e); free(o->phi); free(o->eint); free(o->cs); free(o->ptot); free(o->dphi);
  for (int q = 0; q < 9; q++) {
    free(o->u[q]); free(o->uorg[q]); free(o->src[q]);
    for (int a = 0; a < 3; a++) free(o->flux[a][q]);
  }
  free(o->grvphi); free(o->grvpsi); free(o->gorg1); free(o->gorg2); free(o->lapphi); free(o->hgsrc); free(o->gsrc);
  for (int a = 0; a < 3; a++) { free(o->dir[a][0]); free(o->dir[a][1]); }
  free(o->fbflux);
  free(o->detg1); free(o->idetg1); free(o->sx1); free(o->sini); free(o->cosi); free(o->scot);
  free(o->sinc); free(o->sisin);
  for (int n = 0; n < o->spn; n++) {
    free(o->spc[n]); free(o->spcorg[n]);
    for (int a = 0; a < 3; a++) { free(o->dspc[a][n]); free(o->spcflx[a][n]); }
  }
  free(o);
}

/* compswitch 2 with spn passive scalars (allocations.f90) */
int hmo_set_species(Oracle *o, int spn) {
  if (spn < 0 || spn > MAXSPC || o->spn) return HMO_EBADCFG;
  o->spn = spn;
  for (int n = 0; n < spn; n++) {
    o->spc[n] = zalloc(o->ncell); o->spcorg[n] = zalloc(o->ncell);
    for (int a = 0; a < 3; a++) { o->dspc[a][n] = zalloc(o->ncell); o->spcflx[a][n] = zalloc(o->ncell); }
  }
  return HMO_OK;
}

/* Dirichlet ghost values of face (a, io): 8 + spn planes of 2 x n1 x n2 */
int hmo_set_dirichlet(Oracle *o, int a, int io, const double *vals) {
  int oa[2], q = 0;
  for (int b = 0; b < 3; b++) if (b != a) oa[q++] = b;
  size_t m = (size_t)(8 + o->spn) * 2 * o->n[oa[0]] * o->n[oa[1]];
  if (!o->dir[a][io]) o->dir[a][io] = zalloc(m);
  memcpy(o->dir[a][io], vals, m * sizeof(double));
  return HMO_OK;
}

/* boundary code 10 (fluxboundary3i): the face flux of the inner x3 face */
int hmo_set_flux_boundary(Oracle *o, const double *flux) {
  if (!o->fbflux) o->fbflux = zalloc(9 + MAXSPC);
  memcpy(o->fbflux, flux, (size_t)(9 + o->spn) * sizeof(double));
  return HMO_OK;
}

/* interior values of scalar n (x fastest) */
void hmo_set_spc(Oracle *o, int n, const double *val) {
  size_t q = 0;
  for (int k = 0; k < o->n[2]; k++)
    for (int j = 0; j < o->n[1]; j++)
      for (int i = 0; i < o->n[0]; i++, q++) o->spc[n][IX(o, i, j, k)] = val[q];
}

void hmo_set_times(Oracle *o, double time, double t_end, double dt_out, int outstyle, int endstyle, int tnlim) {
  /* checksetup.f90:202-209 (t_out = min(dt_out,t_end); t_end already in seconds) */
  o->time = time; o->t_end = t_end; o->dt_out = dt_out;
  o->t_out = fmin2(dt_out, t_end);
  o->outstyle = outstyle; o->endstyle = endstyle; o->tnlim = tnlim;
}

void hmo_set_test_mode(Oracle *o) { o->t_out = o->t_end; } /* checksetup.f90:206-209 */

void hmo_set_gravity(Oracle *o, int gravswitch, double HGfac, double hgcfl, double alphagrv, double G, int grktype,
                     int maxtngrv) {
  o->gravswitch = gravswitch; o->HGfac = HGfac; o->hgcfl = hgcfl; o->alphagrv = alphagrv;
  o->G = G; o->grktype = grktype; o->maxtngrv = maxtngrv;
}

/* gridset.f90:46-80 for a uniform Cartesian axis; with gravity the spacing
   arrays are reset to dxi and the two ghost layers are re-accumulated
   (gridset.f90:71-81). */
/* gridset.f90:46-81 from the cell widths dxi(is-2:ie+2) of any Cartesian mesh */
static void make_axis(Oracle *o, int a, double xis, const double *widths, int cart_grav) {
  int n = o->n[a];
  double *x = o->x[a], *xi = o->xi[a], *dx = o->dx[a], *dxi = o->dxi[a], *idx = o->idx[a], *idxi = o->idxi[a];
#define G2(arr, i) arr[(i) + 2]
  for (int i = -2; i <= n + 1; i++) G2(dxi, i) = widths[i + 2];
  for (int i = -1; i <= n + 1; i++) {
    G2(dx, i) = 0.5 * (G2(dxi, i - 1) + G2(dxi, i));
    G2(idxi, i) = 1.0 / G2(dxi, i);
    G2(idx, i) = 1.0 / G2(dx, i);
  }
  G2(x, -1) = xis - G2(dxi, -1) * 0.5;
  G2(x, -2) = G2(x, -1) - G2(dx, -1);
  G2(xi, -1) = xis;
  G2(xi, -2) = xis - G2(dxi, -1);
  for (int i = 0; i <= n + 1; i++) {
    G2(x, i) = G2(x, i - 1) + G2(dx, i);
    G2(xi, i) = G2(xi, i - 1) + G2(dxi, i);
  }
  if (cart_grav) {
    for (int i = -2; i <= n + 1; i++) {
      G2(dx, i) = G2(dxi, i);
      G2(idx, i) = 1.0 / G2(dx, i);
      G2(idxi, i) = 1.0 / G2(dxi, i);
    }
    for (int i = -1; i >= -2; i--) {
      G2(xi, i) = G2(xi, i + 1) - G2(dxi, i);
      G2(x, i) = G2(x, i + 1) - G2(dx, i);
    }
    for (int i = n; i <= n + 1; i++) {
      G2(xi, i) = G2(xi, i - 1) + G2(dxi, i);
      G2(x, i) = G2(x, i - 1) + G2(dx, i);
    }
  }
#undef G2
}

void hmo_make_axis(Oracle *o, int a, double xis, const double *widths) {
  make_axis(o, a, xis, widths, o->gravswitch != 0);
}

/* cell widths dxi(is-2:ie+2) of a geometrical-series mesh (imesh=1):
   utils.f90:351-404 */
static int geometric_widths(int n, double xis, double xie, double xmin, double *w) {
  const double xrmax = 1.05, maxerr = 1e-10;
  double xr = 1.01, xrng = xie - xis, irng = (double)n;
  if (xrng / irng < xmin) return HMO_EBADCFG;
  for (long it = 0; it < 10000000; it++) {
    double fx = (xr - 1.0) * xrng - xmin * (pow(xr, irng) - 1.0);
    double dfx = xrng - irng * xmin * pow(xr, irng - 1.0);
    double xrnew = xr - fx / dfx;
    if (fabs((xrnew - xr) / xr) < maxerr) { xr = xrnew; break; }
    if (xrnew < 1.0) xrnew = 2.0;
    xr = xrnew;
  }
  if (xr > xrmax) return HMO_EBADCFG;
  w[2] = xmin;
  for (int i = 1; i < n; i++) w[i + 2] = w[i + 1] * xr;
  w[1] = w[2];
  w[0] = w[3];
  w[n + 2] = w[n + 1] * xr;
  w[n + 3] = w[n + 1] * xr * xr;
  if (xr - 1.0 < maxerr)
    for (int i = 0; i < n + 4; i++) w[i] = xrng / irng;
  return HMO_OK;
}

int hmo_make_geometric_axis(Oracle *o, int a, double xis, double xie, double xmin) {
  double *w = zalloc((size_t)o->n[a] + 4);
  int rc = geometric_widths(o->n[a], xis, xie, xmin, w);
  if (rc == HMO_OK) hmo_make_axis(o, a, xis, w);
  free(w);
  return rc;
}

/* sin and cos evaluated in quad precision and rounded to double, as
   gridset.f90:376-382 forms sini/cosi with real(..., kind=16) */
static double qsin(double x) { return (double)sinq((__float128)x); }
static double qcos(double x) { return (double)cosq((__float128)x); }

/* Spherical polar grid (crdnt=2) without gravity: r from xi1s to xi1e
   (uniform, or a geometrical series with first width x1min when imesh=1),
   theta over [0, pi] ([0, pi/2] for one theta cell or eq_sym), phi over
   [-pi, pi) (a quarter turn for one phi cell), with the volumetric centres
   of r and theta; gridset.f90:294-423.  Then the metric factors of
   metric.f90:102-151. */
int hmo_make_spherical(Oracle *o, int imesh, double xi1s, double xi1e, double x1min, int eq_sym) {
  const int n1 = o->n[0], n2 = o->n[1], n3 = o->n[2];
  if (n3 > 1 && n3 < 4) return HMO_EBADCFG;
  o->xi1s = xi1s;
  const double pi = acos(-1.0);
  double *w = zalloc((size_t)(n1 > n2 ? (n1 > n3 ? n1 : n3) : (n2 > n3 ? n2 : n3)) + 4);
  /* r */
  if (imesh == 1) {
    int rc = geometric_widths(n1, xi1s, xi1e, x1min, w);
    if (rc) { free(w); return rc; }
  } else {
    for (int i = 0; i < n1 + 4; i++) w[i] = (xi1e - xi1s) / (double)n1;
  }
  make_axis(o, 0, xi1s, w, 0);
  {
    double *x = o->x[0] + 2, *xi = o->xi[0] + 2, *dx = o->dx[0] + 2, *idx = o->idx[0] + 2;
    double *dxi = o->dxi[0] + 2, *idxi = o->idxi[0] + 2;
    for (int i = -1; i <= n1 + 1; i++) { /* :323-329 */
      x[i] = 0.75 * (xi[i] + xi[i - 1]) * (xi[i] * xi[i] + xi[i - 1] * xi[i - 1]) /
             (xi[i] * xi[i] + xi[i] * xi[i - 1] + xi[i - 1] * xi[i - 1]);
      if (i == 0) x[i - 1] = -x[i];
      dx[i] = x[i] - x[i - 1];
      idx[i] = 1.0 / dx[i];
    }
    if (o->gravswitch != 0) { /* :331-343 with the potential's grid equal to the hydro grid (gie = ie) */
      for (int i = n1; i <= n1 + 1; i++) {
        dxi[i] = dxi[i - 1] * dxi[n1 - 1] / dxi[n1 - 2];
        idxi[i] = 1.0 / dxi[i];
        xi[i] = xi[i - 1] + dxi[i];
        x[i] = 0.75 * (xi[i] + xi[i - 1]) * (xi[i] * xi[i] + xi[i - 1] * xi[i - 1]) /
               (xi[i] * xi[i] + xi[i] * xi[i - 1] + xi[i - 1] * xi[i - 1]);
        dx[i] = x[i] - x[i - 1];
        idx[i] = 1.0 / dx[i];
      }
      dx[-2] = dxi[-2];
      for (int i = -2; i <= n1 + 1; i++) { idx[i] = 1.0 / dx[i]; idxi[i] = 1.0 / dxi[i]; }
    }
  }
  /* theta */
  double xi2e = (n2 == 1 || eq_sym) ? pi * 0.5 : pi;
  int jetmp = n2 == 1 ? 1 : n2;
  for (int j = 0; j < n2 + 4; j++) w[j] = xi2e / (double)jetmp;
  make_axis(o, 1, 0.0, w, 0);
  {
    double *x = o->x[1] + 2, *xi = o->xi[1] + 2, *dx = o->dx[1] + 2, *idx = o->idx[1] + 2;
    double *si = o->sini + 2, *ci = o->cosi + 2, *sc = o->sinc + 2;
    for (int j = -2; j <= n2 + 1; j++) { si[j] = qsin(xi[j]); ci[j] = qcos(xi[j]); sc[j] = qsin(x[j]); }
    for (int j = -1; j <= n2 + 1; j++) { /* :385-392 */
      x[j] = (xi[j - 1] * ci[j - 1] - xi[j] * ci[j] + si[j] - si[j - 1]) / (ci[j - 1] - ci[j]);
      if (j == 0) x[j - 1] = -x[j];
      dx[j] = x[j] - x[j - 1];
      idx[j] = 1.0 / dx[j];
    }
  }
  /* phi */
  int ketmp = n3 == 1 ? 4 : n3;
  for (int k = 0; k < n3 + 4; k++) w[k] = (pi - -pi) / (double)ketmp;
  make_axis(o, 2, -pi, w, 0);
  free(w);
  /* metric.f90:102-151 */
  {
    const double *xi = o->xi[0] + 2, *dxi = o->dxi[0] + 2;
    double *g1 = o->detg1 + 2, *ig1 = o->idetg1 + 2, *s1 = o->sx1 + 2;
    for (int i = -1; i <= n1; i++) {
      g1[i] = xi[i] * xi[i];
      ig1[i] = 3.0 / (dxi[i] * (xi[i] * xi[i] + xi[i] * xi[i - 1] + xi[i - 1] * xi[i - 1]));
      s1[i] = 1.5 * (xi[i] + xi[i - 1]) / (xi[i] * xi[i] + xi[i] * xi[i - 1] + xi[i - 1] * xi[i - 1]);
    }
    const double *si = o->sini + 2, *ci = o->cosi + 2;
    const double *xi2 = o->xi[1] + 2;
    double *sc = o->scot + 2, *ss = o->sisin + 2;
    for (int j = -1; j <= n2; j++) {
      sc[j] = (si[j] - si[j - 1]) / (ci[j - 1] - ci[j]);
      ss[j] = (xi2[j] - xi2[j - 1]) / (ci[j - 1] - ci[j]);
    }
  }
  o->fac_k = n3 == 1 ? 4.0 : 1.0;
  o->fac_j = n2 == 1 ? 2.0 : 1.0;
  o->crdnt = 2;
  return HMO_OK;
}

/* Cylindrical grid (crdnt=1) without gravity and with phi unsolved (one
   phi cell): R from xi1s (uniform, or a geometrical series) with the
   volumetric centres sqrt((xi1(i-1)^2 + xi1(i)^2)/2), a quarter turn of
   phi, z from xi3s to xi3e (uniform or geometrical series); then the metric
   of metric.f90:53-100 (gridset.f90:145-292).  A solved phi axis is
   refused: gridset reads an unset width dxi2(js-2) for its ghost centres. */
int hmo_make_cylindrical(Oracle *o, int imesh, double xi1s, double xi1e, double x1min, int kmesh, double xi3s,
                         double xi3e, double x3min) {
  const int n1 = o->n[0], n2 = o->n[1], n3 = o->n[2];
  if (o->gravswitch != 0 || n2 != 1) return HMO_EBADCFG;
  const double pi = acos(-1.0);
  int nmax = n1 > n3 ? n1 : n3;
  double *w = zalloc((size_t)nmax + 4);
  if (imesh == 1) {
    int rc = geometric_widths(n1, xi1s, xi1e, x1min, w);
    if (rc) { free(w); return rc; }
  } else {
    for (int i = 0; i < n1 + 4; i++) w[i] = (xi1e - xi1s) / (double)n1;
  }
  make_axis(o, 0, xi1s, w, 0);
  {
    double *x = o->x[0] + 2, *xi = o->xi[0] + 2, *dx = o->dx[0] + 2, *idx = o->idx[0] + 2;
    for (int i = -1; i <= n1 + 1; i++) { /* :187-193 */
      x[i] = sqrt((xi[i - 1] * xi[i - 1] + xi[i] * xi[i]) * 5e-1);
      if (i == -1) x[i] = -x[i];
      dx[i] = x[i] - x[i - 1];
      idx[i] = 1.0 / dx[i];
    }
  }
  /* phi: four cells of the full turn stand for one (:209-231) */
  for (int j = 0; j < n2 + 4; j++) w[j] = 2.0 * pi / 4.0;
  make_axis(o, 1, 0.0, w, 0);
  /* z */
  if (kmesh == 1 && n3 > 1) {
    int rc = geometric_widths(n3, xi3s, xi3e, x3min, w);
    if (rc) { free(w); return rc; }
  } else {
    for (int k = 0; k < n3 + 4; k++) w[k] = (xi3e - xi3s) / (double)n3;
  }
  make_axis(o, 2, xi3s, w, 0);
  free(w);
  { /* metric.f90:53-100 */
    const double *xi = o->xi[0] + 2;
    double *g1 = o->detg1 + 2, *ig1 = o->idetg1 + 2, *s1 = o->sx1 + 2;
    for (int i = -1; i <= n1; i++) {
      g1[i] = xi[i];
      ig1[i] = 2.0 / (xi[i] * xi[i] - xi[i - 1] * xi[i - 1]);
      s1[i] = 2.0 / (xi[i] + xi[i - 1]);
    }
  }
  o->fac_j = 4.0; /* dvol, sa1, sa3 of one phi cell times four (:92-96) */
  o->fac_k = 1.0;
  o->crdnt = 1;
  return HMO_OK;
}

/* metric arrays of a spherical grid: 0 detg1, 1 idetg1, 2 sx1 (n0+4 each),
   3 sini, 4 cosi, 5 scot, 6 sinc, 7 sisin (n1+4 each) */
int hmo_get_metric(Oracle *o, int which, double *out) {
  const double *src[8] = {o->detg1, o->idetg1, o->sx1, o->sini, o->cosi, o->scot, o->sinc, o->sisin};
  if (which < 0 || which > 7) return -1;
  size_t L = (size_t)o->n[which < 3 ? 0 : 1] + 4;
  memcpy(out, src[which], L * sizeof(double));
  return 0;
}

void hmo_make_uniform_axis(Oracle *o, int a, double xis, double xie) {
  int n = o->n[a];
  double h = (xie - xis) / (double)n;
  double *w = zalloc((size_t)n + 4);
  for (int i = 0; i < n + 4; i++) w[i] = h;
  hmo_make_axis(o, a, xis, w);
  free(w);
}

void hmo_get_axis(Oracle *o, int a, double *x, double *xi, double *dx, double *dxi, double *idx, double *idxi) {
  size_t L = (size_t)o->n[a] + 4;
  memcpy(x, o->x[a], L * 8); memcpy(xi, o->xi[a], L * 8); memcpy(dx, o->dx[a], L * 8);
  memcpy(dxi, o->dxi[a], L * 8); memcpy(idx, o->idx[a], L * 8); memcpy(idxi, o->idxi[a], L * 8);
}

/* ------------------------------------------------------------------------ */
/* EOS (eostype 0)                                                            */

/* eos.f90:846-866 */
static inline double get_eint(const Oracle *o, double etot, double d, double v1, double v2, double v3, double b1,
                              double b2, double b3) {
  double vsq = v1 * v1 + v2 * v2 + v3 * v3;
  double eint = etot - 0.5 * d * vsq;
  if (o->mag_on) {
    double bsq = b1 * b1 + b2 * b2 + b3 * b3;
    eint = eint - 0.5 * bsq;
  }
  return eint;
}

/* eos.f90:351-365 */
static inline double get_cf(double d, double cs, double b1, double b2, double b3) {
  double asq = cs * cs;
  double bb1 = b1 * b1 / d, bb2 = b2 * b2 / d, bb3 = b3 * b3 / d;
  double bbsq = bb1 + bb2 + bb3;
  return sqrt(0.5 * (asq + bbsq + sqrt((asq + bbsq) * (asq + bbsq) - 4.0 * asq * bb1)));
}

static void set_err(Oracle *o, int code, int i, int j, int k) {
  if (!o->err) { o->err = code; o->err_i = i; o->err_j = j; o->err_k = k; }
}

/* eos.f90:742-842 (pressure -> internalenergy), interior cells */
static void pressure(Oracle *o) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  double gm1 = o->gamma - 1.0;
  int bad = 0, bi = 0, bj = 0, bk = 0;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t c = IX(o, i, j, k);
        double ei = get_eint(o, o->e[c], o->d[c], o->v[0][c], o->v[1][c], o->v[2][c], o->b[0][c], o->b[1][c], o->b[2][c]);
        o->eint[c] = ei;
        if (ei <= 0.0) {
#pragma omp critical
          { if (!bad) { bad = 1; bi = i; bj = j; bk = k; } }
        }
        o->p[c] = gm1 * ei;
        o->ptot[c] = o->p[c];
        if (o->mag_on) {
          double bsq = o->b[0][c] * o->b[0][c] + o->b[1][c] * o->b[1][c] + o->b[2][c] * o->b[2][c];
          o->ptot[c] = o->ptot[c] + 0.5 * bsq;
        }
      }
  if (bad) set_err(o, HMO_ENEG_EINT, bi, bj, bk);
}

/* ------------------------------------------------------------------------ */
/* boundary conditions: boundarycondition.f90 codes 0-3                       */

static inline size_t IXa(const Oracle *o, int a, int s, int t1, int t2) {
  /* cell with coordinate s along axis a; (t1,t2) are the other two axes in
     increasing axis order */
  int ijk[3];
  ijk[a] = s;
  int q = 0;
  for (int b = 0; b < 3; b++) if (b != a) ijk[b] = (q++ == 0) ? t1 : t2;
  return IX(o, ijk[0], ijk[1], ijk[2]);
}

static void ghost_energy(Oracle *o, size_t g) {
  /* boundarycondition.f90:222-243 */
  double gm1 = o->gamma - 1.0;
  double b1 = o->b[0][g], b2 = o->b[1][g], b3 = o->b[2][g];
  o->ptot[g] = o->p[g] + 0.5 * (b1 * b1 + b2 * b2 + b3 * b3);
  o->eint[g] = o->p[g] / gm1; /* eos.f90:287-289 */
  double v1 = o->v[0][g], v2 = o->v[1][g], v3 = o->v[2][g];
  o->e[g] = o->eint[g] + 0.5 * (o->d[g] * (v1 * v1 + v2 * v2 + v3 * v3) + b1 * b1 + b2 * b2 + b3 * b3);
}

/* linear extrapolation into the two ghosts beyond the edge cell (code 4/5):
   outer  q(n)   = q(n-1) + (q(n-1)-q(n-2))*dx(n-1)/dx(n-2),
          q(n+1) = q(n)   + (q(n)-q(n-1))*dx(n)/dx(n-1)        (:302-327)
   inner  q(-1)  = q(0)   - (q(1)-q(0))*dx(0)/dx(1),
          q(-2)  = q(-1)  - (q(0)-q(-1))*dx(-1)/dx(0)           (:963-985) */
static void linear_ghosts(const Oracle *o, int a, int io, const double *f, size_t e0, size_t e1, double *g0,
                          double *g1) {
  /* e0: edge cell, e1: the next one inward; g0: near ghost, g1: far ghost */
  const double *DX = o->dx[a] + 2;
  int n = o->n[a];
  if (io == 1) {
    *g0 = f[e0] + (f[e0] - f[e1]) * DX[n - 1] / DX[n - 2];
    *g1 = *g0 + (*g0 - f[e0]) * DX[n] / DX[n - 1];
  } else {
    *g0 = f[e0] - (f[e1] - f[e0]) * DX[0] / DX[1];
    *g1 = *g0 - (f[e0] - *g0) * DX[-1] / DX[0];
  }
}

static void bc_axis(Oracle *o, int a) {
  int n = o->n[a];
  int oa[2], q = 0;
  for (int b = 0; b < 3; b++) if (b != a) oa[q++] = b;
  int n1 = o->n[oa[0]], n2 = o->n[oa[1]];
  size_t area = (size_t)n1 * n2;
  for (int io = 0; io < 2; io++) {
    int bs = o->bc[a][io][0], bv = o->bc[a][io][1];
    for (int t2 = 0; t2 < n2; t2++)
      for (int t1 = 0; t1 < n1; t1++) {
        int edge = io == 0 ? 0 : n - 1;
        size_t ce0 = IXa(o, a, edge, t1, t2), ce1 = IXa(o, a, io == 0 ? 1 : n - 2, t1, t2);
        size_t cnear = IXa(o, a, io == 0 ? -1 : n, t1, t2), cfar = IXa(o, a, io == 0 ? -2 : n + 1, t1, t2);
        size_t fidx = (size_t)t1 + (size_t)n1 * t2;
        if (bs == 4 || bs == 5) {
          double g0, g1;
          linear_ghosts(o, a, io, o->d, ce0, ce1, &g0, &g1);
          if (g1 <= 0.0) g0 = g1 = o->d[ce0];
          o->d[cnear] = g0; o->d[cfar] = g1;
          linear_ghosts(o, a, io, o->p, ce0, ce1, &g0, &g1);
          if (g1 <= 0.0) g0 = g1 = o->p[ce0];
          o->p[cnear] = g0; o->p[cfar] = g1;
          if (o->mag_on) { o->phi[cnear] = o->phi[ce0]; o->phi[cfar] = o->phi[ce0]; }
          for (int ns = 0; ns < o->spn; ns++) { o->spc[ns][cnear] = o->spc[ns][ce0]; o->spc[ns][cfar] = o->spc[ns][ce0]; }
        }
        if (bv == 4 || bv == 5) {
          for (int c = 0; c < 3; c++) {
            double g0, g1;
            linear_ghosts(o, a, io, o->v[c], ce0, ce1, &g0, &g1);
            if (bv == 5 && c == a) {
              /* linear + outgoing: the normal velocity only flows out (:441-468) */
              double plug = io == 1 ? 0.5 + fsign(0.5, o->v[a][ce0]) : 0.5 - fsign(0.5, o->v[a][ce0]);
              g0 = g0 * plug; g1 = g1 * plug;
            }
            o->v[c][cnear] = g0; o->v[c][cfar] = g1;
            if (o->mag_on) {
              linear_ghosts(o, a, io, o->b[c], ce0, ce1, &g0, &g1);
              o->b[c][cnear] = g0; o->b[c][cfar] = g1;
            }
          }
        }
        for (int gl = 0; gl < 2; gl++) {
          /* ghost coordinate and its source cells */
          int g = io == 0 ? -2 + gl : n + gl;       /* is-2,is-1 | ie+1,ie+2 */
          int per = io == 0 ? n - 2 + gl : gl;       /* periodic image */
          int refl = io == 0 ? 1 - gl : n - 1 - gl;  /* reflective image: is+1,is | ie,ie-1 */
          size_t cg = IXa(o, a, g, t1, t2);
          const double *D = o->dir[a][io];
          size_t h = (size_t)gl * area + fidx;
          int ss = -1;
          switch (bs) {
            case 0: ss = per; break;
            case 1: ss = refl; break;
            case 2: case 3: ss = edge; break;
            case 4: case 5: break;
            case 9:
            case 10: /* code 10 never writes its ghosts (boundarycondition.f90:999,1139): they keep the
                        values the host set, given here as for code 9 */
              if (!D) { set_err(o, HMO_EBADCFG, a, io, 0); return; }
              o->d[cg] = D[0 * 2 * area + h]; o->p[cg] = D[1 * 2 * area + h];
              if (o->mag_on) o->phi[cg] = 0.0;
              for (int ns = 0; ns < o->spn; ns++) o->spc[ns][cg] = D[(size_t)(8 + ns) * 2 * area + h];
              break;
            default: set_err(o, HMO_EBADCFG, a, io, 0); return;
          }
          if (ss >= 0) {
            size_t cs_ = IXa(o, a, ss, t1, t2);
            o->d[cg] = o->d[cs_]; o->p[cg] = o->p[cs_];
            for (int ns = 0; ns < o->spn; ns++) o->spc[ns][cg] = o->spc[ns][cs_];
            if (o->mag_on) o->phi[cg] = o->phi[cs_];
          }
          int sv = -1;
          switch (bv) {
            case 0: sv = per; break;
            case 1: sv = refl; break;
            case 2: case 3: sv = edge; break;
            case 4: case 5: break;
            case 9:
            case 10:
              if (!D) { set_err(o, HMO_EBADCFG, a, io, 1); return; }
              for (int c = 0; c < 3; c++) {
                o->v[c][cg] = D[(size_t)(2 + c) * 2 * area + h];
                if (o->mag_on) o->b[c][cg] = D[(size_t)(5 + c) * 2 * area + h];
              }
              break;
            default: set_err(o, HMO_EBADCFG, a, io, 1); return;
          }
          if (sv >= 0) {
            size_t cv = IXa(o, a, sv, t1, t2);
            for (int c = 0; c < 3; c++) {
              double vv = o->v[c][cv];
              if (c == a && bv == 1) vv = -vv;
              if (c == a && bv == 2) {
                if (io == 0) {
                  if (a == 0) vv = fmin2(0.0, vv);                 /* :165 */
                  else vv = vv * (0.5 - fsign(0.5, vv));           /* y/z inner plug */
                } else {
                  vv = vv * (0.5 + fsign(0.5, vv));                /* :388-390 */
                }
              }
              o->v[c][cg] = vv;
              if (o->mag_on) {
                double bb = o->b[c][cv];
                if (c == a && bv == 1) bb = -bb;
                o->b[c][cg] = bb;
              }
            }
          }
        }
        for (int gl = 0; gl < 2; gl++) {
          int g = io == 0 ? -2 + gl : n + gl;
          ghost_energy(o, IXa(o, a, g, t1, t2));
        }
      }
  }
}

static void boundarycondition(Oracle *o) {
  bc_axis(o, 0);                 /* x1 is always applied (boundarycondition.f90:51) */
  if (o->solve[1]) bc_axis(o, 1); /* :523 */
  if (o->solve[2]) bc_axis(o, 2);
}

/* ------------------------------------------------------------------------ */
/* limiters: fluxlimiter.f90:40-56 (minmod), 58-75 (modified_mc)            */

static inline double minmod(const double u[3], const double dx[2]) {
  double x = 1.4 * (u[2] - u[1]) * dx[1];
  double y = 1.4 * (u[1] - u[0]) * dx[0];
  double z = (u[2] - u[0]) * dx[0] * dx[1] / (dx[0] + dx[1]);
  double s = fsign(1.0, x);
  double m = fabs(x);
  m = fmin2(m, s * y);
  m = fmin2(m, s * z);
  return s * fmax2(0.0, m);
}

static inline double modified_mc(const double u[3], const double x[3], const double xi[2]) {
  double cf = (x[2] - x[1]) / (xi[1] - x[1]);
  double cb = (x[1] - x[0]) / (x[1] - xi[0]);
  double top = (u[1] - u[0]) * (x[2] - x[1]) / (x[1] - x[0]);
  double bot = u[2] - u[1];
  double sig = fsign(1.0, bot);
  double m = sig * 0.5 * (bot + top);
  m = fmin2(m, sig * cf * bot);
  m = fmin2(m, sig * cb * top);
  return sig * fmax2(0.0, m) / (x[2] - x[1]);
}

/* ------------------------------------------------------------------------ */
/* interpolation.f90:49-484                                                   */

static void interpolation(Oracle *o) {
  if (o->limiter == 0) return; /* flat: slopes stay zero (interpolation.f90:42-45) */
  for (int a = 0; a < 3; a++) {
    if (!o->solve[a]) continue;
    int n = o->n[a];
    int oa[2], q = 0;
    for (int b = 0; b < 3; b++) if (b != a) oa[q++] = b;
    int n1 = o->n[oa[0]], n2 = o->n[oa[1]];
    const double *X = o->x[a] + 2, *XI = o->xi[a] + 2, *IDX = o->idx[a] + 2;
#pragma omp parallel for collapse(2) schedule(static)
    for (int t2 = 0; t2 < n2; t2++)
      for (int t1 = 0; t1 < n1; t1++)
        for (int s = -1; s <= n; s++) {
          size_t cm = IXa(o, a, s - 1, t1, t2), c0 = IXa(o, a, s, t1, t2), cp = IXa(o, a, s + 1, t1, t2);
          double dx2[2] = {IDX[s], IDX[s + 1]};
          double xx[3] = {X[s - 1], X[s], X[s + 1]};
          double xxi[2] = {XI[s - 1], XI[s]};
          double hl = X[s] - XI[s - 1], hr = XI[s] - X[s];
          double uu[3], du, L[NSLOPE], R[NSLOPE];
          int nsl = o->mag_on ? NSLOPE : S_B1;
          for (int sl = 0; sl < nsl; sl++) {
            switch (sl) {
              case S_D: uu[0] = o->d[cm]; uu[1] = o->d[c0]; uu[2] = o->d[cp]; break;
              case S_E: uu[0] = o->e[cm]; uu[1] = o->e[c0]; uu[2] = o->e[cp]; break;
              case S_M1: case S_M2: case S_M3: {
                int vc = sl - S_M1;
                uu[0] = o->d[cm] * o->v[vc][cm]; uu[1] = o->d[c0] * o->v[vc][c0]; uu[2] = o->d[cp] * o->v[vc][cp];
              } break;
              default: {
                int bcmp = sl - S_B1;
                uu[0] = o->b[bcmp][cm]; uu[1] = o->b[bcmp][c0]; uu[2] = o->b[bcmp][cp];
              }
            }
            du = o->limiter == 1 ? minmod(uu, dx2) : modified_mc(uu, xx, xxi);
            o->slope[a][sl][c0] = du;
            L[sl] = uu[1] - hl * du;
            R[sl] = uu[1] + hr * du;
          }
          /* interpolation.f90:135-141: scalar slopes, never zeroed below */
          for (int ns = 0; ns < o->spn; ns++) {
            uu[0] = o->spc[ns][cm]; uu[1] = o->spc[ns][c0]; uu[2] = o->spc[ns][cp];
            o->dspc[a][ns][c0] = o->limiter == 1 ? minmod(uu, dx2) : modified_mc(uu, xx, xxi);
          }
          double eintl = L[S_E] - 0.5 * (L[S_M1] * L[S_M1] + L[S_M2] * L[S_M2] + L[S_M3] * L[S_M3]) / L[S_D];
          double eintr = R[S_E] - 0.5 * (R[S_M1] * R[S_M1] + R[S_M2] * R[S_M2] + R[S_M3] * R[S_M3]) / R[S_D];
          if (o->mag_on) {
            eintl = eintl - 0.5 * (L[S_B1] * L[S_B1] + L[S_B2] * L[S_B2] + L[S_B3] * L[S_B3]);
            eintr = eintr - 0.5 * (R[S_B1] * R[S_B1] + R[S_B2] * R[S_B2] + R[S_B3] * R[S_B3]);
          }
          double em = o->eint[cm], e0 = o->eint[c0], ep = o->eint[cp];
          if (eintl >= fmax2(em, e0) || eintl <= fmin2(em, e0) || eintr >= fmax2(e0, ep) || eintr <= fmin2(e0, ep)) {
            for (int sl = 0; sl < NSLOPE; sl++) o->slope[a][sl][c0] = 0.0;
            o->dphi[c0] = 0.0;
          }
        }
  }
}

/* ------------------------------------------------------------------------ */
/* hlldflux.f90:19-179                                                        */

static void hlldflux(double f[9], double cfl, double cfr, double v1l, double v1r, double v2l, double v2r, double v3l,
                     double v3r, double dl, double dr, double el, double er, double ptl, double ptr, double b1l,
                     double b1r, double b2l, double b2r, double b3l, double b3r, double phil, double phir,
                     double ch) {
  double b1 = 0.5 * ((b1l + b1r) - (phir - phil) / ch);
  double phi = 0.5 * ((phil + phir) - (b1r - b1l) * ch);
  double sl = fmin2(fmin2(v1r - cfr, v1l - cfl), 0.0);
  double sr = fmax2(fmax2(v1r + cfr, v1l + cfl), 0.0);
  double sm = ((sr - v1r) * dr * v1r - (sl - v1l) * dl * v1l - ptr + ptl) / ((sr - v1r) * dr - (sl - v1l) * dl);
  double dla = dl * (sl - v1l) / (sl - sm);
  double dra = dr * (sr - v1r) / (sr - sm);
  double sla = sm - fabs(b1) / sqrt(dla);
  double sra = sm + fabs(b1) / sqrt(dra);
  double pta = ((sr - v1r) * dr * ptl - (sl - v1l) * dl * ptr + dl * dr * (sr - v1r) * (sl - v1l) * (v1r - v1l)) /
               ((sr - v1r) * dr - (sl - v1l) * dl);
  double v2la = v2l - b1 * b2l * (sm - v1l) / (dl * (sl - v1l) * (sl - sm) - b1 * b1);
  double v2ra = v2r - b1 * b2r * (sm - v1r) / (dr * (sr - v1r) * (sr - sm) - b1 * b1);
  double v3la = v3l - b1 * b3l * (sm - v1l) / (dl * (sl - v1l) * (sl - sm) - b1 * b1);
  double v3ra = v3r - b1 * b3r * (sm - v1r) / (dr * (sr - v1r) * (sr - sm) - b1 * b1);
  double b2la = b2l * (dl * (sl - v1l) * (sl - v1l) - b1 * b1) / (dl * (sl - v1l) * (sl - sm) - b1 * b1);
  double b2ra = b2r * (dr * (sr - v1r) * (sr - v1r) - b1 * b1) / (dr * (sr - v1r) * (sr - sm) - b1 * b1);
  double b3la = b3l * (dl * (sl - v1l) * (sl - v1l) - b1 * b1) / (dl * (sl - v1l) * (sl - sm) - b1 * b1);
  double b3ra = b3r * (dr * (sr - v1r) * (sr - v1r) - b1 * b1) / (dr * (sr - v1r) * (sr - sm) - b1 * b1);
  double ela = ((sl - v1l) * el - ptl * v1l + pta * sm +
                b1 * ((v1l * b1 + v2l * b2l + v3l * b3l) - (sm * b1 + v2la * b2la + v3la * b3la))) /
               (sl - sm);
  double era = ((sr - v1r) * er - ptr * v1r + pta * sm +
                b1 * ((v1r * b1 + v2r * b2r + v3r * b3r) - (sm * b1 + v2ra * b2ra + v3ra * b3ra))) /
               (sr - sm);
  double s1 = fsign(1.0, b1);
  double v2aa = (sqrt(dla) * v2la + sqrt(dra) * v2ra + (b2ra - b2la) * s1) / (sqrt(dla) + sqrt(dra));
  double v3aa = (sqrt(dla) * v3la + sqrt(dra) * v3ra + (b3ra - b3la) * s1) / (sqrt(dla) + sqrt(dra));
  double b2aa = (sqrt(dla) * b2ra + sqrt(dra) * b2la + sqrt(dla * dra) * (v2ra - v2la) * s1) / (sqrt(dla) + sqrt(dra));
  double b3aa = (sqrt(dla) * b3ra + sqrt(dra) * b3la + sqrt(dla * dra) * (v3ra - v3la) * s1) / (sqrt(dla) + sqrt(dra));
  double eraa = era + s1 * sqrt(dra) * ((v2ra * b2ra + v3ra * b3ra) - (v2aa * b2aa + v3aa * b3aa));
  double elaa = ela - s1 * sqrt(dla) * ((v2la * b2la + v3la * b3la) - (v2aa * b2aa + v3aa * b3aa));
  double signsm = fsign(0.5, sm);
  double sortsla = 0.5 + fsign(0.5, sla);
  double sortsra = 0.5 + fsign(0.5, -sra);
  double sortslr = 0.5 - fsign(0.5, sla * sra);
  dla = (0.5 + signsm) * dla + (0.5 - signsm) * dra;
  v2la = sortsla * v2la + sortslr * v2aa + sortsra * v2ra;
  v3la = sortsla * v3la + sortslr * v3aa + sortsra * v3ra;
  b2la = sortsla * b2la + sortslr * b2aa + sortsra * b2ra;
  b3la = sortsla * b3la + sortslr * b3aa + sortsra * b3ra;
  ela = sortsla * ela + (0.5 - fsign(0.5, sla * sm)) * elaa + (0.5 + fsign(0.5, -(sm * sra))) * eraa +
        (0.5 - fsign(0.5, sra)) * era;
  /* fstar (hlldflux.f90:156-179) */
  double d = dla, v1 = sm, v2 = v2la, v3 = v3la, bb2 = b2la, bb3 = b3la, e = ela, p = pta;
  f[0] = d * v1;
  f[1] = d * v1 * v1 + p - b1 * b1;
  f[2] = d * v1 * v2 - b1 * bb2;
  f[3] = d * v1 * v3 - b1 * bb3;
  f[4] = (e + p) * v1 - b1 * (v1 * b1 + v2 * bb2 + v3 * bb3);
  f[5] = phi;
  f[6] = bb2 * v1 - b1 * v2;
  f[7] = bb3 * v1 - b1 * v3;
  f[8] = ch * ch * b1;
}

/* numflux.f90:46-563 */
/* fluxboundary3i (fluxboundary.f90:42-87, called at numflux.f90:566): the
   flux through the inner x3 face replaced by the host-given wind flux */
static void fluxboundary(Oracle *o) {
  if (o->bc[2][0][0] != 10 || !o->solve[2]) return;
  if (!o->fbflux) { set_err(o, HMO_EBADCFG, 2, 0, 10); return; }
  for (int j = 0; j < o->n[1]; j++)
    for (int i = 0; i < o->n[0]; i++) {
      size_t f = IX(o, i, j, -1);
      for (int q = 0; q < 9; q++) o->flux[2][q][f] = o->fbflux[q];
      for (int ns = 0; ns < o->spn; ns++) o->spcflx[2][ns][f] = o->fbflux[9 + ns];
    }
}

static void numflux(Oracle *o) {
  interpolation(o);
  double gam = o->gamma, gm1 = o->gamma - 1.0;
  for (int a = 0; a < 3; a++) {
    if (!o->solve[a]) continue;
    int n = o->n[a];
    int oa[2], q = 0;
    for (int b = 0; b < 3; b++) if (b != a) oa[q++] = b;
    int n1 = o->n[oa[0]], n2 = o->n[oa[1]];
    const double *X = o->x[a] + 2, *XI = o->xi[a] + 2;
    /* component rotation: normal, first tangent, second tangent */
    int cn = a, c1 = (a + 1) % 3, c2 = (a + 2) % 3;
    int bad = 0, bi = 0, bj = 0, bk = 0;
#pragma omp parallel for collapse(2) schedule(static)
    for (int t2 = 0; t2 < n2; t2++)
      for (int t1 = 0; t1 < n1; t1++)
        for (int s = -1; s <= n - 1; s++) {
          size_t L = IXa(o, a, s, t1, t2), R = IXa(o, a, s + 1, t1, t2);
          double dx1 = XI[s] - X[s], dx2 = X[s + 1] - XI[s];
          double *const *sp = o->slope[a];
          double dl = o->d[L] + dx1 * sp[S_D][L];
          double dr = o->d[R] - dx2 * sp[S_D][R];
          double el = o->e[L] + dx1 * sp[S_E][L];
          double er = o->e[R] - dx2 * sp[S_E][R];
          double v1l = (o->d[L] * o->v[cn][L] + dx1 * sp[S_M1 + cn][L]) / dl;
          double v1r = (o->d[R] * o->v[cn][R] - dx2 * sp[S_M1 + cn][R]) / dr;
          double v2l = (o->d[L] * o->v[c1][L] + dx1 * sp[S_M1 + c1][L]) / dl;
          double v2r = (o->d[R] * o->v[c1][R] - dx2 * sp[S_M1 + c1][R]) / dr;
          double v3l = (o->d[L] * o->v[c2][L] + dx1 * sp[S_M1 + c2][L]) / dl;
          double v3r = (o->d[R] * o->v[c2][R] - dx2 * sp[S_M1 + c2][R]) / dr;
          double b1l = 0, b1r = 0, b2l = 0, b2r = 0, b3l = 0, b3r = 0, phil = 0, phir = 0;
          if (o->mag_on) {
            b1l = o->b[cn][L] + dx1 * sp[S_B1 + cn][L];
            b1r = o->b[cn][R] - dx2 * sp[S_B1 + cn][R];
            b2l = o->b[c1][L] + dx1 * sp[S_B1 + c1][L];
            b2r = o->b[c1][R] - dx2 * sp[S_B1 + c1][R];
            b3l = o->b[c2][L] + dx1 * sp[S_B1 + c2][L];
            b3r = o->b[c2][R] - dx2 * sp[S_B1 + c2][R];
            phil = o->phi[L] + dx1 * o->dphi[L];
            phir = o->phi[R] - dx2 * o->dphi[R];
          }
          double eil = get_eint(o, el, dl, v1l, v2l, v3l, b1l, b2l, b3l);
          double eir = get_eint(o, er, dr, v1r, v2r, v3r, b1r, b2r, b3r);
          double erl = 0.0, err = 0.0;
          /* eos_p_cs (eos.f90:195-242) with erad present */
          int ierr = 0;
          double ptl = 0, ptr = 0, csl = 0, csr = 0;
          if (eil <= 0.0 || dl <= 0.0) ierr = 1;
          else {
            ptl = gm1 * eil;
            double cs2 = gam * ptl / dl;
            cs2 = cs2 + 4.0 * erl / (9.0 * dl);
            csl = sqrt(cs2);
          }
          if (eir <= 0.0 || dr <= 0.0) ierr = 1;
          else {
            ptr = gm1 * eir;
            double cs2 = gam * ptr / dr;
            cs2 = cs2 + 4.0 * err / (9.0 * dr);
            csr = sqrt(cs2);
          }
          if (ierr) {
#pragma omp critical
            {
              if (!bad) {
                bad = 1;
                int ijk[3]; ijk[a] = s; ijk[oa[0]] = t1; ijk[oa[1]] = t2;
                bi = ijk[0]; bj = ijk[1]; bk = ijk[2];
              }
            }
            continue;
          }
          ptl = ptl + 0.5 * (b1l * b1l + b2l * b2l + b3l * b3l);
          ptr = ptr + 0.5 * (b1r * b1r + b2r * b2r + b3r * b3r);
          double cfl = get_cf(dl, csl, b1l, b2l, b3l);
          double cfr = get_cf(dr, csr, b1r, b2r, b3r);
          double f[9];
          hlldflux(f, cfl, cfr, v1l, v1r, v2l, v2r, v3l, v3r, dl, dr, el, er, ptl, ptr, b1l, b1r, b2l, b2r, b3l,
                   b3r, phil, phir, o->ch);
          double *const *F = o->flux[a];
          F[ICNT][L] = f[0];
          F[IMO1 + cn][L] = f[1];
          F[IMO1 + c1][L] = f[2];
          F[IMO1 + c2][L] = f[3];
          F[IENE][L] = f[4];
          if (o->mag_on) {
            F[IMG1 + cn][L] = f[5];
            F[IMG1 + c1][L] = f[6];
            F[IMG1 + c2][L] = f[7];
            if (o->dim > 1) F[I9WV][L] = f[8];
          }
          if (o->spn) {
            /* numflux.f90:200-212: upwinded face fractions renormalised to sum 1 */
            double spl[MAXSPC], spr[MAXSPC], suml = 0.0, sumr = 0.0;
            for (int ns = 0; ns < o->spn; ns++) {
              spl[ns] = o->spc[ns][L] + dx1 * o->dspc[a][ns][L];
              spr[ns] = o->spc[ns][R] - dx2 * o->dspc[a][ns][R];
            }
            for (int ns = 0; ns < o->spn; ns++) suml = suml + spl[ns]; /* Fortran sum(), left to right */
            for (int ns = 0; ns < o->spn; ns++) sumr = sumr + spr[ns];
            double sg = fsign(0.5, f[0]);
            double fix = 1.0 / (suml * (0.5 + sg) + sumr * (0.5 - sg));
            for (int ns = 0; ns < o->spn; ns++)
              o->spcflx[a][ns][L] = fix * f[0] * (spl[ns] * (0.5 + sg) + spr[ns] * (0.5 - sg));
          }
        }
    if (bad) set_err(o, HMO_ENEG_EINT, bi, bj, bk);
  }
  fluxboundary(o);
}

/* ------------------------------------------------------------------------ */
/* source.f90:14-85,177-228 (Cartesian)                                       */

static void source(Oracle *o) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  int grav = o->gravswitch == 2 || o->gravswitch == 3;
  if (grav) {
    /* get_fieldforce(totphi=grvphi, d) */
    const double *dx1 = o->dx[0] + 2, *idx1 = o->idx[0] + 2;
    const double *dx2 = o->dx[1] + 2, *idx2 = o->idx[1] + 2;
    const double *dx3 = o->dx[2] + 2, *idx3 = o->idx[2] + 2;
    const double *ph = o->grvphi;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          size_t c = IX(o, i, j, k);
          double dd = o->d[c];
          o->grv[0][c] = -((dx1[i] * idx1[i + 1] * ph[IX(o, i + 1, j, k)] - dx1[i + 1] * idx1[i] * ph[IX(o, i - 1, j, k)]) /
                               (dx1[i] + dx1[i + 1]) +
                           (dx1[i + 1] - dx1[i]) * idx1[i] * idx1[i + 1] * ph[c]) * dd;
          o->grv[1][c] = -((dx2[j] * idx2[j + 1] * ph[IX(o, i, j + 1, k)] - dx2[j + 1] * idx2[j] * ph[IX(o, i, j - 1, k)]) /
                               (dx2[j] + dx2[j + 1]) +
                           (dx2[j + 1] - dx2[j]) * idx2[j] * idx2[j + 1] * ph[c]) * dd;
          o->grv[2][c] = -((dx3[k] * idx3[k + 1] * ph[IX(o, i, j, k + 1)] - dx3[k + 1] * idx3[k] * ph[IX(o, i, j, k - 1)]) /
                               (dx3[k] + dx3[k + 1]) +
                           (dx3[k + 1] - dx3[k]) * idx3[k] * idx3[k + 1] * ph[c]) * dd;
        }
  }
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t c = IX(o, i, j, k);
        for (int q = 0; q < 9; q++) o->src[q][c] = 0.0;
        if (o->crdnt == 1) {
          /* cylindrical geometric terms (source.f90:88-111) */
          const double d = o->d[c], v1 = o->v[0][c], v2 = o->v[1][c], v3 = o->v[2][c], pt = o->ptot[c];
          const double s1 = o->sx1[i + 2];
          o->src[IMO1][c] = (d * v2 * v2 + pt) * s1;
          o->src[IMO2][c] = -(d * v1 * v2 * s1);
          if (o->mag_on) {
            const double b1 = o->b[0][c], b2 = o->b[1][c], b3 = o->b[2][c];
            o->src[IMO1][c] = o->src[IMO1][c] - b2 * b2 * s1;
            o->src[IMO2][c] = o->src[IMO2][c] + b1 * b2 * s1;
            o->src[IMG2][c] = (b1 * v3 - b3 * v1) * s1;
          }
          continue;
        }
        if (o->crdnt == 2) {
          /* spherical geometric terms (source.f90:113-143; no gravity here) */
          const double d = o->d[c], v1 = o->v[0][c], v2 = o->v[1][c], v3 = o->v[2][c], pt = o->ptot[c];
          const double s1 = o->sx1[i + 2], sc = o->scot[j + 2];
          o->src[IMO1][c] = (d * (v2 * v2 + v3 * v3) + 2.0 * pt) * s1;
          o->src[IMO2][c] = ny > 1 ? (-(d * v1 * v2) + (d * (v3 * v3) + pt) * sc) * s1 : 0.0;
          o->src[IMO3][c] = (-(d * v1 * v3) - d * v2 * v3 * sc) * s1;
          if (o->mag_on) {
            const double b1 = o->b[0][c], b2 = o->b[1][c], b3 = o->b[2][c];
            o->src[IMO1][c] = o->src[IMO1][c] - (b2 * b2 + b3 * b3) * s1;
            o->src[IMO2][c] = o->src[IMO2][c] + (b1 * b2 - b3 * b3 * sc) * s1;
            o->src[IMO3][c] = o->src[IMO3][c] + (b1 * b3 + b2 * b3 * sc) * s1;
            o->src[IMG2][c] = (b2 * v1 - b1 * v2) * s1;
            o->src[IMG3][c] = ((v2 * b3 - b2 * v3) * sc - (b1 * v3 - b3 * v1)) * s1;
          }
          if (grav) { /* source.f90:145-150 */
            const double g1 = o->grv[0][c], g2 = o->grv[1][c], g3 = o->grv[2][c], si = o->sisin[j + 2];
            o->src[IMO1][c] = o->src[IMO1][c] + g1;
            o->src[IMO2][c] = o->src[IMO2][c] + g2 * s1;
            o->src[IMO3][c] = o->src[IMO3][c] + g3 * s1 * si;
            o->src[IENE][c] = g1 * v1 + g2 * v2 * s1 + g3 * v3 * s1 * si;
          }
          continue;
        }
        if (grav) {
          o->src[IMO1][c] = o->grv[0][c];
          o->src[IMO2][c] = o->grv[1][c];
          o->src[IMO3][c] = o->grv[2][c];
          o->src[IENE][c] = o->grv[0][c] * o->v[0][c] + o->grv[1][c] * o->v[1][c] + o->grv[2][c] * o->v[2][c];
        }
      }
}

/* ------------------------------------------------------------------------ */
/* rungekutta.f90:16-98,146-232                                               */

static void get_runge_coeff(int iter, int type, double *faco, double *fact, double *facn) {
  if (type == 3) {
    if (iter == 1) { *faco = 1.0; *fact = 1.0; *facn = 0.0; }
    else if (iter == 2) { *faco = 0.75; *fact = 0.25; *facn = *fact; }
    else { *faco = 1.0 / 3.0; *fact = 2.0 / 3.0; *facn = *fact; }
  } else if (type == 2) {
    if (iter == 1) { *faco = 1.0; *fact = 1.0; *facn = 0.0; }
    else { *faco = 0.5; *fact = 0.5; *facn = *fact; }
  } else { *faco = 1.0; *fact = 1.0; *facn = 0.0; }
}

static void primitive(Oracle *o) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t c = IX(o, i, j, k);
        o->d[c] = o->u[ICNT][c];
        o->v[0][c] = o->u[IMO1][c] / o->d[c];
        o->v[1][c] = o->u[IMO2][c] / o->d[c];
        o->v[2][c] = o->u[IMO3][c] / o->d[c];
        o->e[c] = o->u[IENE][c];
        if (o->mag_on) {
          o->b[0][c] = o->u[IMG1][c];
          o->b[1][c] = o->u[IMG2][c];
          o->b[2][c] = o->u[IMG3][c];
          if (o->dim > 1) o->phi[c] = o->u[I9WV][c];
        }
      }
  pressure(o);
}

static void rungekutta(Oracle *o) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  double faco, fact, facn;
  get_runge_coeff(o->rungen, o->rktype, &faco, &fact, &facn);
  const double *idxi1 = o->idxi[0] + 2, *idxi2 = o->idxi[1] + 2, *idxi3 = o->idxi[2] + 2;
  double dt = o->dt;
  for (int q = 0; q < o->nvar; q++) {
    double *U = o->u[q], *UO = o->uorg[q], *F1 = o->flux[0][q], *F2 = o->flux[1][q], *F3 = o->flux[2][q];
    const double *S = o->src[q];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          size_t c = IX(o, i, j, k);
          if (o->rungen == 1) UO[c] = U[c];
          if (o->crdnt == 1) {
            /* idetg1 (detg1 = xi1) along R; idetg2 = idxi2/x1 (never used: phi is unsolved); idetg3 = idxi3 */
            const double *g1 = o->detg1 + 2;
            double id2 = 1.0 / o->x[0][i + 2] * idxi2[j];
            U[c] = faco * UO[c] + facn * U[c] +
                   fact * dt *
                       (o->idetg1[i + 2] * (g1[i - 1] * F1[IX(o, i - 1, j, k)] - g1[i] * F1[c]) +
                        id2 * (1.0 * F2[IX(o, i, j - 1, k)] - 1.0 * F2[c]) +
                        idxi3[k] * (F3[IX(o, i, j, k - 1)] - F3[c]) + S[c]);
            continue;
          }
          if (o->crdnt == 2) {
            /* idetg1, idetg2 = sx1/(cos(theta_-)-cos(theta_+)), idetg3 (metric.f90:105-130) */
            const double *g1 = o->detg1 + 2, *si = o->sini + 2, *ci = o->cosi + 2, *s1 = o->sx1 + 2;
            const double *dxi2 = o->dxi[1] + 2;
            double id2 = 1.0 / (-ci[j] + ci[j - 1]) * s1[i];
            double id3 = id2 * dxi2[j] * idxi3[k] / o->fac_k;
            U[c] = faco * UO[c] + facn * U[c] +
                   fact * dt *
                       (o->idetg1[i + 2] * (g1[i - 1] * F1[IX(o, i - 1, j, k)] - g1[i] * F1[c]) +
                        id2 * (si[j - 1] * F2[IX(o, i, j - 1, k)] - si[j] * F2[c]) +
                        id3 * (F3[IX(o, i, j, k - 1)] - F3[c]) + S[c]);
            continue;
          }
          U[c] = faco * UO[c] + facn * U[c] +
                 fact * dt *
                     (idxi1[i] * (1.0 * F1[IX(o, i - 1, j, k)] - 1.0 * F1[c]) +
                      idxi2[j] * (1.0 * F2[IX(o, i, j - 1, k)] - 1.0 * F2[c]) +
                      idxi3[k] * (F3[IX(o, i, j, k - 1)] - F3[c]) + S[c]);
        }
  }
  /* rungekutta.f90:61-86: scalars from the new density */
  for (int ns = 0; ns < o->spn; ns++) {
    double *X = o->spc[ns], *XO = o->spcorg[ns];
    double *F1 = o->spcflx[0][ns], *F2 = o->spcflx[1][ns], *F3 = o->spcflx[2][ns];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          size_t c = IX(o, i, j, k);
          if (o->rungen == 1) XO[c] = X[c] * o->uorg[ICNT][c];
          X[c] = (faco * XO[c] + facn * X[c] * o->d[c] +
                  fact * dt *
                      (idxi1[i] * (1.0 * F1[IX(o, i - 1, j, k)] - 1.0 * F1[c]) +
                       idxi2[j] * (1.0 * F2[IX(o, i, j - 1, k)] - 1.0 * F2[c]) +
                       idxi3[k] * (F3[IX(o, i, j, k - 1)] - F3[c]))) /
                 o->u[ICNT][c];
        }
  }
  primitive(o);
}

/* hydro.f90:15-52 */
int hmo_hydro_step(Oracle *o) {
  for (o->rungen = 1; o->rungen <= o->rktype; o->rungen++) {
    boundarycondition(o);
    numflux(o);
    if (o->err) return o->err;
    source(o);
    rungekutta(o);
    if (o->err) return o->err;
  }
  return o->err;
}

/* ------------------------------------------------------------------------ */
/* timestep.f90:15-183                                                        */

int hmo_timestep(Oracle *o) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  double gm1 = o->gamma - 1.0, gam = o->gamma;
  double off[3] = {o->solve[0] ? 1.0 : 0.0, o->solve[1] ? 1.0 : 0.0, o->solve[2] ? 1.0 : 0.0};
  const double *dxi1 = o->dxi[0] + 2, *dxi2 = o->dxi[1] + 2, *dxi3 = o->dxi[2] + 2;
  double cfmax = 0.0, dtimin = INFINITY;
  int bad = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(max : cfmax) reduction(min : dtimin)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t c = IX(o, i, j, k);
        double d = o->d[c], ei = o->eint[c];
        if (ei <= 0.0 || d <= 0.0) { bad = 1; continue; }
        o->p[c] = gm1 * ei;
        o->cs[c] = sqrt(gam * o->p[c] / d);
        double cf1, cf2, cf3;
        if (o->mag_on) {
          double b1 = o->b[0][c], b2 = o->b[1][c], b3 = o->b[2][c];
          cf1 = get_cf(d, o->cs[c], b1, b2, b3) + fabs(o->v[0][c]);
          cf2 = get_cf(d, o->cs[c], b2, b1, b3) + fabs(o->v[1][c]);
          cf3 = get_cf(d, o->cs[c], b3, b1, b2) + fabs(o->v[2][c]);
        } else {
          cf1 = o->cs[c] + fabs(o->v[0][c]);
          cf2 = o->cs[c] + fabs(o->v[1][c]);
          cf3 = o->cs[c] + fabs(o->v[2][c]);
        }
        /* metric.f90:45-48 */
        double dvol = dxi1[i] * dxi2[j] * dxi3[k];
        double sa1m = dxi2[j] * dxi3[k], sa1p = dxi2[j] * dxi3[k];
        double sa2m = dxi1[i] * dxi3[k], sa2p = dxi1[i] * dxi3[k];
        double sa3m = dxi1[i] * dxi2[j], sa3p = dxi1[i] * dxi2[j];
        if (o->crdnt == 1) { /* metric.f90:80-96, one phi cell: dvol, sa1, sa3 times four */
          const double *xi = o->xi[0] + 2;
          const double a = xi[i], b = xi[i - 1], f4 = o->fac_j;
          dvol = 0.5 * (a * a - b * b) * dxi2[j] * dxi3[k] * f4;
          sa1m = b * dxi2[j] * dxi3[k] * f4;
          sa1p = a * dxi2[j] * dxi3[k] * f4;
          sa2m = dxi1[i] * dxi3[k];
          sa2p = sa2m;
          sa3p = 0.5 * (a * a - b * b) * dxi2[j] * f4;
          sa3m = sa3p;
        }
        if (o->crdnt == 2) { /* metric.f90:117-130 */
          const double *xi = o->xi[0] + 2, *si = o->sini + 2, *ci = o->cosi + 2;
          const double fj = o->fac_j, fk = o->fac_k;
          const double a = xi[i], b = xi[i - 1];
          dvol = (a * a * a - b * b * b) / 3.0 * (ci[j - 1] - ci[j]) * dxi3[k] * fj * fk;
          sa1p = 0.5 * (a * a) * (ci[j - 1] - ci[j]) * dxi3[k] * fj * fk;
          sa1m = 0.5 * (b * b) * (ci[j - 1] - ci[j]) * dxi3[k] * fj * fk;
          sa2p = 0.5 * si[j] * (a * a - b * b) * dxi3[k] * fk;
          sa2m = 0.5 * si[j - 1] * (a * a - b * b) * dxi3[k] * fk;
          sa3p = 0.5 * (a * a - b * b) * dxi2[j] * fj;
          sa3m = sa3p;
        }
        double dti = dvol / (cf1 * off[0] * (sa1m + sa1p) + cf2 * off[1] * (sa2m + sa2p) + cf3 * off[2] * (sa3m + sa3p));
        double cm = fmax2(fmax2(cf1, cf2), cf3);
        cfmax = fmax2(cfmax, cm);
        dtimin = fmin2(dtimin, dti);
      }
  if (bad) { set_err(o, HMO_ENEG_EINT, -1, -1, -1); return o->err; }
  o->cfmax = cfmax;
  double dt = o->courant * dtimin;
  if (o->outstyle == 1) {
    double t_ref = o->t_out;
    if (o->endstyle == 1) t_ref = fmin2(o->t_out, o->t_end);
    if (t_ref - o->time - dt > 0.0 && t_ref - o->time - 2.0 * dt < 0.0) dt = 0.5 * (t_ref - o->time);
    else dt = fmin2(dt, o->t_out - o->time);
  }
  if (o->endstyle == 1) dt = fmin2(dt, o->t_end - o->time);
  o->dt = dt;
  o->ch = cfmax;
  if (o->gravswitch == 3) {
    o->cgrav = o->HGfac * cfmax;
    if (o->maxtngrv > 0) o->cgrav = fmin2(o->cgrav, o->hgcfl * o->dtg_unit * (double)o->maxtngrv / dt);
    o->dtgrav = fmin2(dt, o->hgcfl * o->dtg_unit / o->cgrav);
  }
  return 0;
}

/* source.f90:239-260 */
void hmo_phidamp(Oracle *o) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  double f = exp(-o->alpha9wave * o->courant);
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) o->phi[IX(o, i, j, k)] = o->phi[IX(o, i, j, k)] * f;
}

/* ------------------------------------------------------------------------ */
/* hyperbolic self-gravity, Cartesian form                                    */

/* distance from the origin of the centre of cell (i,j,k) */
static inline double rdist(const Oracle *o, int i, int j, int k) {
  double x = o->x[0][i + 2], y = o->x[1][j + 2], z = o->x[2][k + 2];
  return sqrt(x * x + y * y + z * z);
}

/* 7-point coefficients: the Cartesian counterpart of
   gravity_hyperbolic.f90:385-406 (radial weights -> 1); outer faces of a
   non-periodic axis use the Robin condition phi ~ 1/r folded into c0 as in
   gravity_hyperbolic.f90:400-404. */
static void lap_coeffs(const Oracle *o, int i, int j, int k, double c[7], double *cnorm) {
  const double *dx1 = o->dx[0] + 2, *dx2 = o->dx[1] + 2, *dx3 = o->dx[2] + 2;
  const double *idx1 = o->idx[0] + 2, *idx2 = o->idx[1] + 2, *idx3 = o->idx[2] + 2;
  const double *dxi1 = o->dxi[0] + 2, *dxi2 = o->dxi[1] + 2, *dxi3 = o->dxi[2] + 2;
  double c0 = -((idx1[i] + idx1[i + 1]) * dxi2[j] * dxi3[k] + (idx2[j] + idx2[j + 1]) * dxi1[i] * dxi3[k] +
                (idx3[k] + idx3[k + 1]) * dxi1[i] * dxi2[j]);
  double cxm = dxi2[j] * dxi3[k] / dx1[i], cxp = dxi2[j] * dxi3[k] / dx1[i + 1];
  double cym = dxi1[i] * dxi3[k] / dx2[j], cyp = dxi1[i] * dxi3[k] / dx2[j + 1];
  double czm = dxi1[i] * dxi2[j] / dx3[k], czp = dxi1[i] * dxi2[j] / dx3[k + 1];
  int ijk[3] = {i, j, k};
  double *cm[3] = {&cxm, &cym, &czm}, *cp[3] = {&cxp, &cyp, &czp};
  for (int a = 0; a < 3; a++) {
    int n = o->n[a];
    int per = o->bc[a][0][0] == 0;
    if (per) continue;
    if (ijk[a] == n - 1) {
      int g[3] = {i, j, k}; g[a] = n;
      c0 = c0 + *cp[a] * rdist(o, i, j, k) / rdist(o, g[0], g[1], g[2]);
      *cp[a] = 0.0;
    }
    if (ijk[a] == 0) {
      int g[3] = {i, j, k}; g[a] = -1;
      c0 = c0 + *cm[a] * rdist(o, i, j, k) / rdist(o, g[0], g[1], g[2]);
      *cm[a] = 0.0;
    }
  }
  c[0] = c0; c[1] = cxm; c[2] = cxp; c[3] = cym; c[4] = cyp; c[5] = czm; c[6] = czp;
  *cnorm = dxi1[i] * dxi2[j] * dxi3[k];
}

/* lap_coeff(0..3) and the normalisation lap_coeff(-1) at coefficient index
   (i,j,k), i, j, k >= -1, of a spherical grid (setup_grv_hyperbolic,
   gravity_hyperbolic.f90:336-400): the axisymmetric (r, theta) form for one
   phi cell, the 3-D form otherwise; the Robin condition at the outer radius
   (gbtype 1), Neumann at the last theta face, and the inner-radius term when
   the grid does not reach r = 0. */
static void lap_coeffs_sph(const Oracle *o, int i, int j, int k, double c[5]) {
  const double *x1 = o->x[0] + 2, *xi1 = o->xi[0] + 2, *dx1 = o->dx[0] + 2, *dxi1 = o->dxi[0] + 2;
  const double *dx2 = o->dx[1] + 2, *dxi2 = o->dxi[1] + 2;
  const double *dx3 = o->dx[2] + 2, *dxi3 = o->dxi[2] + 2, *idx3 = o->idx[2] + 2;
  const double *sinc = o->sinc + 2, *sini = o->sini + 2;
  const int gie = o->n[0] - 1, gje = o->n[1] - 1;
  const double a = xi1[i], b = xi1[i - 1];
  if (o->n[2] == 1) { /* :336-363 */
    c[0] = -((a * a / dx1[i + 1] + b * b / dx1[i]) * sinc[j] * dxi2[j] +
             (sini[j] / dx2[j + 1] + sini[j - 1] / dx2[j]) * dxi1[i]);
    c[1] = a * a * sinc[j] * dxi2[j] / dx1[i + 1];
    c[2] = sini[j] * dxi1[i] / dx2[j + 1];
    c[3] = 0.0;
    if (i == 0 && o->xi1s > 0.0) c[0] = c[0] + b * b * sinc[j] * dxi2[j] / dx1[i];
    if (i == gie) { c[0] = c[0] + c[1] * x1[i] / x1[i + 1]; c[1] = 0.0; }
    if (j == gje) { c[0] = c[0] + c[2]; c[2] = 0.0; }
    c[4] = x1[i] * x1[i] * sinc[j] * dxi1[i] * dxi2[j];
  } else { /* :367-400 */
    c[0] = -((a * a / dx1[i + 1] + b * b / dx1[i]) * sinc[j] * dxi2[j] * dxi3[k] +
             (sini[j] / dx2[j + 1] + sini[j - 1] / dx2[j]) * dxi1[i] * dxi3[k] +
             (idx3[k] + idx3[k + 1]) * dxi1[i] * dxi2[j]);
    c[1] = a * a * sinc[j] * dxi2[j] * dxi3[k] / dx1[i + 1];
    c[2] = sini[j] * dxi1[i] * dxi3[k] / dx2[j + 1];
    c[3] = dxi1[i] * dxi2[j] / dx3[k + 1];
    if (j == gje) { c[0] = c[0] + c[2]; c[2] = 0.0; }
    if (i == 0 && o->xi1s > 0.0) c[0] = c[0] + b * b * sinc[j] * dxi2[j] * dxi3[k] / dx1[i];
    if (i == gie) { c[0] = c[0] + c[1] * x1[i] / x1[i + 1]; c[1] = 0.0; }
    c[4] = x1[i] * x1[i] * sinc[j] * dxi1[i] * dxi2[j] * dxi3[k];
  }
}

static inline int wrap(int s, int n, int per) {
  if (!per) return s;
  if (s < 0) return s + n;
  if (s >= n) return s - n;
  return s;
}

/* gravity_hyperbolic.f90:230-280 */
static void get_lapphi_hgsrc(Oracle *o) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  double fourpiG = 4.0 * M_PI * o->G;
  int px = o->bc[0][0][0] == 0, py = o->bc[1][0][0] == 0, pz = o->bc[2][0][0] == 0;
  const double *ph = o->grvphi;
  if (o->crdnt == 2) { /* :243-270 with the spherical coefficients; ghosts as hg_boundary_conditions left them */
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          double c[5], cxm[5], cym[5], czm[5];
          lap_coeffs_sph(o, i, j, k, c);
          lap_coeffs_sph(o, i - 1, j, k, cxm);
          size_t cc = IX(o, i, j, k);
          double lap = c[0] * ph[cc];
          lap = lap + cxm[1] * ph[IX(o, i - 1, j, k)];
          lap = lap + c[1] * ph[IX(o, i + 1, j, k)];
          if (ny > 1) {
            lap_coeffs_sph(o, i, j - 1, k, cym);
            lap = lap + cym[2] * ph[IX(o, i, j - 1, k)];
            lap = lap + c[2] * ph[IX(o, i, j + 1, k)];
          }
          if (nz > 1) {
            lap_coeffs_sph(o, i, j, k - 1, czm);
            lap = lap + czm[3] * ph[IX(o, i, j, wrap(k - 1, nz, pz))];
            lap = lap + c[3] * ph[IX(o, i, j, wrap(k + 1, nz, pz))];
          }
          o->lapphi[cc] = lap / c[4];
          o->hgsrc[cc] = fourpiG * o->gsrc[cc];
        }
    return;
  }
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        double c[7], cn;
        lap_coeffs(o, i, j, k, c, &cn);
        size_t cc = IX(o, i, j, k);
        double lap = c[0] * ph[cc];
        lap = lap + c[1] * ph[IX(o, wrap(i - 1, nx, px), j, k)];
        lap = lap + c[2] * ph[IX(o, wrap(i + 1, nx, px), j, k)];
        lap = lap + c[3] * ph[IX(o, i, wrap(j - 1, ny, py), k)];
        lap = lap + c[4] * ph[IX(o, i, wrap(j + 1, ny, py), k)];
        lap = lap + c[5] * ph[IX(o, i, j, wrap(k - 1, nz, pz))];
        lap = lap + c[6] * ph[IX(o, i, j, wrap(k + 1, nz, pz))];
        o->lapphi[cc] = lap / cn;
        o->hgsrc[cc] = fourpiG * o->gsrc[cc];
      }
}

/* ghost potential for the hydro gravity force: the Robin image
   phi_g = phi_edge * r_edge / r_g of gravity_hyperbolic.f90:190, applied on
   every non-periodic face; periodic faces copy the opposite edge. */
static void hg_boundary_conditions(Oracle *o) {
  if (o->crdnt == 2) { /* gravity_hyperbolic.f90:186-216, gbtype 1 */
    const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
    const double *x1 = o->x[0] + 2;
    double *ph = o->grvphi;
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++) {
        ph[IX(o, -1, j, k)] = ph[IX(o, 0, j, k)];
        ph[IX(o, nx, j, k)] = ph[IX(o, nx - 1, j, k)] * x1[nx - 1] / x1[nx];
      }
    for (int k = 0; k < nz; k++)
      for (int i = -1; i <= nx; i++) {
        ph[IX(o, i, -1, k)] = ph[IX(o, i, 0, k)];
        ph[IX(o, i, ny, k)] = ph[IX(o, i, ny - 1, k)];
      }
    if (nz > 1)
      for (int j = -1; j <= ny; j++)
        for (int i = -1; i <= nx; i++) {
          ph[IX(o, i, j, -1)] = ph[IX(o, i, j, nz - 1)];
          ph[IX(o, i, j, nz)] = ph[IX(o, i, j, 0)];
        }
    return;
  }
  for (int a = 0; a < 3; a++) {
    int n = o->n[a];
    int per = o->bc[a][0][0] == 0;
    int oa[2], q = 0;
    for (int b = 0; b < 3; b++) if (b != a) oa[q++] = b;
    for (int t2 = 0; t2 < o->n[oa[1]]; t2++)
      for (int t1 = 0; t1 < o->n[oa[0]]; t1++) {
        int gi[3], ei[3];
        /* inner ghost */
        gi[a] = -1; gi[oa[0]] = t1; gi[oa[1]] = t2;
        ei[a] = per ? n - 1 : 0; ei[oa[0]] = t1; ei[oa[1]] = t2;
        size_t g = IX(o, gi[0], gi[1], gi[2]), s = IX(o, ei[0], ei[1], ei[2]);
        if (per) o->grvphi[g] = o->grvphi[s];
        else o->grvphi[g] = o->grvphi[s] * rdist(o, ei[0], ei[1], ei[2]) / rdist(o, gi[0], gi[1], gi[2]);
        /* outer ghost */
        gi[a] = n; ei[a] = per ? 0 : n - 1;
        g = IX(o, gi[0], gi[1], gi[2]); s = IX(o, ei[0], ei[1], ei[2]);
        if (per) o->grvphi[g] = o->grvphi[s];
        else o->grvphi[g] = o->grvphi[s] * rdist(o, ei[0], ei[1], ei[2]) / rdist(o, gi[0], gi[1], gi[2]);
      }
  }
}

/* gravity_hyperbolic.f90:61-125 */
static void hyperbolic_gravity_step(Oracle *o, double cgrav_now, double cgrav_old, double dtg) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  for (int g = 1; g <= o->grktype; g++) {
    double faco, fact, facn;
    get_runge_coeff(g, o->grktype, &faco, &fact, &facn);
    get_lapphi_hgsrc(o);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          size_t c = IX(o, i, j, k);
          if (g == 1) { o->gorg1[c] = o->grvphi[c]; o->gorg2[c] = o->grvpsi[c]; }
          double ph = faco * o->gorg1[c] + facn * o->grvphi[c] + fact * dtg * cgrav_now * o->grvpsi[c];
          double ps = faco * o->gorg2[c] + facn * o->grvpsi[c] + fact * dtg * cgrav_now * (o->lapphi[c] - o->hgsrc[c]);
          o->grvphi[c] = ph;
          o->grvpsi[c] = ps;
        }
  }
  double damp = exp(-(1.0 - cgrav_old / cgrav_now + o->alphagrv * o->hgcfl));
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) o->grvpsi[IX(o, i, j, k)] = o->grvpsi[IX(o, i, j, k)] * damp;
}

/* gravity.f90:18-64 (tn>0, gravswitch 3) -> gravity_hyperbolic.f90:19-50 */
int hmo_gravity(Oracle *o) {
  if (o->gravswitch != 3) return 0;
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) o->gsrc[IX(o, i, j, k)] = o->d[IX(o, i, j, k)]; /* gravity.f90:136-150 */
  if (o->tn == 0) { hg_boundary_conditions(o); return 0; } /* grav_init_other */
  int tngrav = (int)ceil((o->time + o->dt - o->grvtime) / o->dtgrav);
  double dtg = (o->time + o->dt - o->grvtime) / (double)tngrav;
  o->dtgrav = dtg;
  for (int l = 0; l < tngrav; l++) {
    hyperbolic_gravity_step(o, o->cgrav, o->cgrav_old, dtg);
    o->grvtime = o->grvtime + dtg;
    o->cgrav_old = o->cgrav;
  }
  hg_boundary_conditions(o);
  return 0;
}

/* tools.f90:160-183: dtg_unit = min over cells of dtgrav_cell(cgrav=1) */
void hmo_gravity_setup(Oracle *o, double cgrav_old) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  double off[3] = {o->solve[0] ? 1.0 : 0.0, o->solve[1] ? 1.0 : 0.0, o->solve[2] ? 1.0 : 0.0};
  const double *dxi1 = o->dxi[0] + 2, *dxi2 = o->dxi[1] + 2, *dxi3 = o->dxi[2] + 2;
  double m = INFINITY;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        double dvol = dxi1[i] * dxi2[j] * dxi3[k];
        double s1 = dxi2[j] * dxi3[k] + dxi2[j] * dxi3[k];
        double s2 = dxi1[i] * dxi3[k] + dxi1[i] * dxi3[k];
        double s3 = dxi1[i] * dxi2[j] + dxi1[i] * dxi2[j];
        if (o->crdnt == 2) { /* dtgrav_cell with metric.f90:117-130 */
          const double *xi = o->xi[0] + 2, *si = o->sini + 2, *ci = o->cosi + 2;
          const double fj = o->fac_j, fk = o->fac_k, a = xi[i], b = xi[i - 1];
          dvol = (a * a * a - b * b * b) / 3.0 * (ci[j - 1] - ci[j]) * dxi3[k] * fj * fk;
          s1 = 0.5 * (b * b) * (ci[j - 1] - ci[j]) * dxi3[k] * fj * fk +
               0.5 * (a * a) * (ci[j - 1] - ci[j]) * dxi3[k] * fj * fk;
          s2 = 0.5 * si[j - 1] * (a * a - b * b) * dxi3[k] * fk + 0.5 * si[j] * (a * a - b * b) * dxi3[k] * fk;
          s3 = 0.5 * (a * a - b * b) * dxi2[j] * fj + 0.5 * (a * a - b * b) * dxi2[j] * fj;
        }
        double v = dvol / (1.0 * (off[0] * s1 + off[1] * s2 + off[2] * s3));
        m = fmin2(m, v);
      }
  o->dtg_unit = m;
  o->cgrav_old = cgrav_old;
  o->grvtime = o->time;
}

/* ------------------------------------------------------------------------ */
/* initial state and main loop                                                */

/* initialcondition.f90:132-141 + the start-up sequence of hormone.f90:94-100
   (boundarycondition, conserve, pressure).  Inputs are interior arrays of
   n0*n1*n2 doubles, x fastest. */
void hmo_set_prims(Oracle *o, const double *d, const double *p, const double *v1, const double *v2, const double *v3,
                   const double *b1, const double *b2, const double *b3, const double *phi) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  double gm1 = o->gamma - 1.0;
  size_t q = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++, q++) {
        size_t c = IX(o, i, j, k);
        o->d[c] = d[q]; o->p[c] = p[q];
        o->v[0][c] = v1[q]; o->v[1][c] = v2[q]; o->v[2][c] = v3[q];
        o->b[0][c] = b1 ? b1[q] : 0.0; o->b[1][c] = b2 ? b2[q] : 0.0; o->b[2][c] = b3 ? b3[q] : 0.0;
        o->phi[c] = phi ? phi[q] : 0.0;
        o->eint[c] = o->p[c] / gm1;
        double vv = o->v[0][c] * o->v[0][c] + o->v[1][c] * o->v[1][c] + o->v[2][c] * o->v[2][c];
        double bb = o->b[0][c] * o->b[0][c] + o->b[1][c] * o->b[1][c] + o->b[2][c] * o->b[2][c];
        o->e[c] = o->eint[c] + o->d[c] * 0.5 * vv + 0.5 * bb;
      }
  boundarycondition(o);
  /* conserve.f90:13-50 */
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t c = IX(o, i, j, k);
        o->u[ICNT][c] = o->d[c];
        o->u[IMO1][c] = o->d[c] * o->v[0][c];
        o->u[IMO2][c] = o->d[c] * o->v[1][c];
        o->u[IMO3][c] = o->d[c] * o->v[2][c];
        o->u[IENE][c] = o->e[c];
        if (o->mag_on) {
          o->u[IMG1][c] = o->b[0][c]; o->u[IMG2][c] = o->b[1][c]; o->u[IMG3][c] = o->b[2][c];
          if (o->dim > 1) o->u[I9WV][c] = o->phi[c];
        }
      }
  pressure(o);
  o->tn = 0;
}

void hmo_set_grvphi(Oracle *o, const double *phi, const double *psi) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  size_t q = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++, q++) {
        o->grvphi[IX(o, i, j, k)] = phi[q];
        o->grvpsi[IX(o, i, j, k)] = psi ? psi[q] : 0.0;
      }
}

/* one pass of hormone.f90:126-155; returns 1 when the run has ended */
int hmo_step(Oracle *o) {
  int rc = hmo_timestep(o);
  if (rc) return rc;
  hmo_gravity(o);
  rc = hmo_hydro_step(o);
  if (rc) return rc;
  if (o->mag_on && o->dim > 1) hmo_phidamp(o);
  o->time = o->time + o->dt;
  o->tn = o->tn + 1;
  if (o->endstyle == 1 && o->time >= o->t_end) return 1;
  if (o->endstyle == 2 && o->tn >= o->tnlim) return 1;
  if (o->outstyle == 1 && o->time >= o->t_out) o->t_out = o->t_out + o->dt_out;
  return 0;
}

/* initial timestep + gravity (hormone.f90:107-113), then the loop */
int hmo_start(Oracle *o) {
  int rc = hmo_timestep(o);
  if (rc) return rc;
  if (o->gravswitch == 3) hmo_gravity(o);
  return 0;
}

int hmo_run(Oracle *o, int max_steps) {
  for (int s = 0; s < max_steps; s++) {
    int rc = hmo_step(o);
    if (rc < 0) return rc;
    if (rc == 1) return 1;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* accessors                                                                  */

/* which: 0 d,1 p,2 e,3 v1,4 v2,5 v3,6 b1,7 b2,8 b3,9 phi,10 eint,11 cs,
   12 grvphi, 13 grvpsi, 20+q u(q), 30+n spc(n) */
int hmo_get(Oracle *o, int which, double *out) {
  const int nx = o->n[0], ny = o->n[1], nz = o->n[2];
  const double *src;
  switch (which) {
    case 0: src = o->d; break;
    case 1: src = o->p; break;
    case 2: src = o->e; break;
    case 3: case 4: case 5: src = o->v[which - 3]; break;
    case 6: case 7: case 8: src = o->b[which - 6]; break;
    case 9: src = o->phi; break;
    case 10: src = o->eint; break;
    case 11: src = o->cs; break;
    case 12: src = o->grvphi; break;
    case 13: src = o->grvpsi; break;
    default:
      if (which >= 20 && which < 29) { src = o->u[which - 20]; break; }
      if (which >= 30 && which < 30 + o->spn) { src = o->spc[which - 30]; break; }
      return -1;
  }
  size_t q = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++, q++) out[q] = src[IX(o, i, j, k)];
  return 0;
}

void hmo_scalars(Oracle *o, double *out) {
  out[0] = o->time; out[1] = o->dt; out[2] = o->ch; out[3] = o->cfmax; out[4] = o->cgrav; out[5] = o->dtgrav;
  out[6] = o->dtg_unit; out[7] = o->grvtime; out[8] = o->cgrav_old; out[9] = (double)o->tn; out[10] = o->t_out;
}

void hmo_set_scalars(Oracle *o, double time, int tn, double grvtime, double cgrav_old) {
  o->time = time; o->tn = tn; o->grvtime = grvtime; o->cgrav_old = cgrav_old;
}

void hmo_error(Oracle *o, int *out) { out[0] = o->err; out[1] = o->err_i; out[2] = o->err_j; out[3] = o->err_k; }

int hmo_nvar(Oracle *o) { return o->nvar; }
