/* host_driver.c -- a C host of the library, built with a C compiler against
 * include/hormone_gpu.h: what a Fortran ISO_C_BINDING shim binds.
 *
 *   host_driver layout            one line per struct field: "<struct>.<field> <offset>",
 *                                 then "sizeof <struct> <bytes>" (no library calls)
 *   host_driver run IN OUT        HORMONE's step loop (src/main/hormone.f90:107-179:
 *                                 timestep once, then timestep -> hydro_step ->
 *                                 phidamp -> time += dt until t_end) through the C ABI
 *
 * IN (little-endian, written by tests/test_host_driver.py):
 *   int32 n[3], bc[12], rktype, grktype, limiter, mag_on, gravswitch, maxtngrv,
 *         outstyle, endstyle, nvar, glm
 *   float64 gamma, courant, alpha9wave, HGfac, hgcfl, alphagrv, G, t_out, dt_out, t_end
 *   per axis: x, xi, dx, dxi, idx, idxi (n+4 values each)
 *   u (nvar planes), then the primitives d, v1, v2, v3, e, b1, b2, b3, phi
 *   (each n0*n1*n2 values, x fastest)
 * OUT: int32 tn, float64 time, then u and the nine primitives as above.
 */
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hormone_gpu.h"

#define F(s, f) printf(#s "." #f " %zu\n", offsetof(s, f))

static int layout(void) {
  F(hmn_grid, n);
  F(hmn_grid, ghost);
  F(hmn_grid, bc);
  F(hmn_grid, x);
  F(hmn_grid, xi);
  F(hmn_grid, dx);
  F(hmn_grid, dxi);
  F(hmn_grid, idx);
  F(hmn_grid, idxi);
  printf("sizeof hmn_grid %zu\n", sizeof(hmn_grid));
  F(hmn_params, gamma);
  F(hmn_params, courant);
  F(hmn_params, alpha9wave);
  F(hmn_params, HGfac);
  F(hmn_params, hgcfl);
  F(hmn_params, alphagrv);
  F(hmn_params, G);
  F(hmn_params, rktype);
  F(hmn_params, grktype);
  F(hmn_params, limiter);
  F(hmn_params, mag_on);
  F(hmn_params, gravswitch);
  F(hmn_params, maxtngrv);
  F(hmn_params, outstyle);
  F(hmn_params, endstyle);
  F(hmn_params, precision);
  F(hmn_params, nspc);
  printf("sizeof hmn_params %zu\n", sizeof(hmn_params));
  F(hmn_metric, detg1);
  F(hmn_metric, idetg1);
  F(hmn_metric, sx1);
  F(hmn_metric, sini);
  F(hmn_metric, cosi);
  F(hmn_metric, scot);
  F(hmn_metric, sinc);
  F(hmn_metric, sisin);
  printf("sizeof hmn_metric %zu\n", sizeof(hmn_metric));
  return 0;
}

#ifndef HMN_LAYOUT_ONLY
static void rd(void* p, size_t sz, size_t n, FILE* f) {
  if (fread(p, sz, n, f) != n) {
    fprintf(stderr, "host_driver: short input\n");
    exit(2);
  }
}

#define CK(call)                                                      \
  do {                                                                \
    int rc_ = (call);                                                 \
    if (rc_ != HMN_OK) {                                              \
      fprintf(stderr, "host_driver: %s returned %d\n", #call, rc_);   \
      return 3;                                                       \
    }                                                                 \
  } while (0)

static int run(const char* in, const char* out) {
  FILE* f = fopen(in, "rb");
  if (!f) return 2;
  int n[3], bc[12], iv[10];
  double dv[10];
  rd(n, sizeof(int), 3, f);
  rd(bc, sizeof(int), 12, f);
  rd(iv, sizeof(int), 10, f);
  rd(dv, sizeof(double), 10, f);
  hmn_grid g;
  memset(&g, 0, sizeof(g));
  double* axes[3][6];
  for (int a = 0; a < 3; a++) {
    g.n[a] = n[a];
    for (int k = 0; k < 6; k++) {
      axes[a][k] = (double*)malloc(sizeof(double) * (size_t)(n[a] + 4));
      rd(axes[a][k], sizeof(double), (size_t)(n[a] + 4), f);
    }
    g.x[a] = axes[a][0];
    g.xi[a] = axes[a][1];
    g.dx[a] = axes[a][2];
    g.dxi[a] = axes[a][3];
    g.idx[a] = axes[a][4];
    g.idxi[a] = axes[a][5];
  }
  g.ghost = 0;
  memcpy(g.bc, bc, sizeof(g.bc));
  hmn_params p;
  memset(&p, 0, sizeof(p));
  p.rktype = iv[0];
  p.grktype = iv[1];
  p.limiter = iv[2];
  p.mag_on = iv[3];
  p.gravswitch = iv[4];
  p.maxtngrv = iv[5];
  p.outstyle = iv[6];
  p.endstyle = iv[7];
  const int nvar = iv[8], glm = iv[9];
  p.gamma = dv[0];
  p.courant = dv[1];
  p.alpha9wave = dv[2];
  p.HGfac = dv[3];
  p.hgcfl = dv[4];
  p.alphagrv = dv[5];
  p.G = dv[6];
  double t_out = dv[7];
  const double dt_out = dv[8], t_end = dv[9];
  const size_t cells = (size_t)n[0] * n[1] * n[2];
  double* u = (double*)malloc(sizeof(double) * cells * nvar);
  rd(u, sizeof(double), cells * nvar, f);
  double* prim[9];
  for (int q = 0; q < 9; q++) {
    prim[q] = (double*)malloc(sizeof(double) * cells);
    rd(prim[q], sizeof(double), cells, f);
  }
  fclose(f);

  hmn_ctx* ctx = NULL;
  CK(hmn_create(&g, &p, &ctx));
  CK(hmn_upload(ctx, u, (const double* const*)prim, NULL, NULL));
  double time = 0.0, dt = 0.0, ch = 0.0;
  int tn = 0;
  CK(hmn_timestep(ctx, time, t_out, t_end, &dt, &ch)); /* hormone.f90:107 */
  for (;;) {                                           /* hormone.f90:124-179 */
    CK(hmn_timestep(ctx, time, t_out, t_end, &dt, &ch));
    CK(hmn_hydro_step(ctx));
    if (glm) CK(hmn_phidamp(ctx));
    time = time + dt;
    tn += 1;
    if (p.endstyle == 1 && time >= t_end) break;
    if (p.outstyle == 1 && time >= t_out) t_out = t_out + dt_out;
    if (tn > 10000000) return 4;
  }
  CK(hmn_download(ctx, u, prim, NULL, NULL));
  CK(hmn_destroy(ctx));
  FILE* o = fopen(out, "wb");
  if (!o) return 2;
  fwrite(&tn, sizeof(int), 1, o);
  fwrite(&time, sizeof(double), 1, o);
  fwrite(u, sizeof(double), cells * nvar, o);
  for (int q = 0; q < 9; q++) fwrite(prim[q], sizeof(double), cells, o);
  fclose(o);
  return 0;
}
#endif

int main(int argc, char** argv) {
  if (argc >= 2 && strcmp(argv[1], "layout") == 0) return layout();
#ifndef HMN_LAYOUT_ONLY
  if (argc >= 4 && strcmp(argv[1], "run") == 0) return run(argv[2], argv[3]);
#endif
  fprintf(stderr, "usage: host_driver layout | run IN OUT\n");
  return 1;
}
