// hmn_internal.h -- structures shared by the C-ABI layer and the kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "hmn_tma.cuh"

namespace hmn {

// Per-axis geometry, each array indexed [c+2] for c in [-2, n+1] (the
// Fortran range is-2..ie+2).  Derived once on the host from the grid arrays
// the caller passes, with the same single IEEE operations the reference
// performs inside its loops, so that reading them is bit-equivalent to
// recomputing them.
struct AxisGeo {
  const double* x;     // cell centres
  const double* dx;    // centre spacing dx(c) = x(c)-x(c-1) as the grid defines it
  const double* idx;   // 1/dx(c)
  const double* dxi;   // cell width
  const double* idxi;  // 1/dxi(c)
  const double* hl;    // x(c) - xi(c-1): centre to left face
  const double* hr;    // xi(c) - x(c): centre to right face
  const double* mcf;   // (x(c+1)-x(c)) / (xi(c)-x(c))      modified_mc cf
  const double* mcb;   // (x(c)-x(c-1)) / (x(c)-xi(c-1))    modified_mc cb
  const double* ga;    // x(c+1) - x(c)
  const double* gb;    // x(c) - x(c-1)
  const double* isum;  // idx(c) + idx(c+1)                  minmod denominator
  // reciprocal forms used only by the mixed-precision stage (division-free limiters)
  const double* rga;   // 1 / ga
  const double* gab;   // ga / gb
  const double* risum; // 1 / isum
};
constexpr int kGeoArrays = 15;

// Curvilinear coordinates: spherical polar (crd 2; r, theta, phi as axes
// 1-3) or cylindrical with one phi cell (crd 1; R, phi, z).  The 1-D
// factors of the metric (metric.f90:53-151), each at offset +2 like the
// axis arrays.  The 2-D and 3-D factors of the reference (idetg2, idetg3,
// dvol, sa1..3) are formed from them per cell in the reference's operation
// order.  on = 0 for Cartesian grids; the theta arrays are unset for crd 1.
struct SphGeo {
  int on;
  int crd;
  double fac_j, fac_k;   // spherical: 2 for a single theta cell, 4 for a single phi cell, else 1;
                         // cylindrical: fac_j = 4 (dvol, sa1, sa3 of the single phi cell)
  const double* detg1;   // weight of the r flux through the high face of cell i: xi1^2 (xi1 cylindrical)
  const double* idetg1;  // 3 / (dxi1 (xi1(i)^2 + xi1(i) xi1(i-1) + xi1(i-1)^2)) (2 / (xi1(i)^2 - xi1(i-1)^2))
  const double* sx1;     // 1.5 (xi1(i) + xi1(i-1)) / (same sum of squares) (2 / (xi1(i) + xi1(i-1)))
  const double* vr;      // (xi1(i)^3 - xi1(i-1)^3) / 3: radial factor of dvol
  const double* hr2;     // 0.5 xi1(i)^2: radial factor of sa1
  const double* ar2;     // xi1(i)^2 - xi1(i-1)^2: radial factor of sa2, sa3
  const double* sini;    // sin(theta) at the high face of cell j (detg2)
  const double* ra2;     // 1 / (cos(theta)(j-1) - cos(theta)(j)): theta factor of idetg2
  const double* cd;      // cos(theta)(j-1) - cos(theta)(j): theta factor of dvol, sa1
  const double* scot;    // (sin(j) - sin(j-1)) / (cos(j-1) - cos(j))
  const double* sisin;   // (xi2(j) - xi2(j-1)) / (cos(j-1) - cos(j)): phi factor of the gravity source
};

struct GridDev {
  int n[3];
  int solve[3];
  int bc[3][2][2];  // [axis][inner,outer][scalar,vector]
  AxisGeo g[3];
  // slab decomposition along z: the two cell layers beyond the low / high z
  // face come from the neighbouring slab (primitive planes x 2 layers x
  // nx*ny, filled by the caller's exchange) instead of the boundary codes;
  // nullptr on a physical face; zwrap[io] = 1 where the face is the grid's
  // periodic z boundary, whose ghosts take the boundary condition's form
  // (energies rebuilt from the pressure) rather than the interior values
  const double* zhalo[2];
  int zwrap[2];
  // the same for the gravitational potential: the one layer (nx*ny) beyond
  // the low / high z face, from the neighbouring slab, or nullptr
  const double* ghalo[2];
  // boundary code 9 (Dirichlet): ghost values of face [axis][inner,outer],
  // 8 + nspc planes (d, p, v1..3, b1..3, scalars) x 2 layers x face cells
  // (layer l at coordinate -2+l inner, n+l outer; the other two axes in
  // increasing order, the lower one fastest)
  const double* dir[3][2];
  // boundary code 10 at the inner z face: the flux through that face
  // (9 conserved slots, then the scalars), or nullptr
  const double* fb;
  SphGeo sph;
  // 1 where, for every cell index c of the three axes, idx(c) = RN(1/dx(c))
  // and dx(c) lies in [2^-500, 2^501) (checked on the host): the quotients
  // by dx may then be corrected from idx without forming the reciprocal
  int idx_rn;
};

// Device-resident scalars of one simulation: the CFL reduction slots, the
// step's dt/ch and the first error seen by any kernel.
struct DevScalars {
  unsigned long long min_dti_bits;  // atomicMin over bit patterns of dti > 0
  unsigned long long cfmax_bits;    // atomicMax over bit patterns of cf >= 0
  double time, t_out, t_end;
  double dt, ch, cfmax;
  double cgrav, dtgrav, dtg_unit;
  double courant, HGfac, hgcfl;
  int outstyle, endstyle, gravswitch, maxtngrv;
  int err_code, err_i, err_j, err_k;
  int done;  // set by advance_kernel once time >= t_end; later launches of hmn_run skip their work
  int tn;
};

// Arguments of one fused RK stage launch (hmn_kernels.cu: stage_kernel).
struct StageArgs {
  const double* pin;    // primitive planes of the state entering the stage (stencil source)
  double* pout;         // primitive planes of the state leaving the stage
  const double* uorg;   // RK base state U^n (pointwise)
  const double* ucur;   // state entering this stage (pointwise)
  double* uout;         // state leaving this stage
  const double* gphi;   // gravitational potential (interior planes) or nullptr
  DevScalars* sc;       // dt, ch, errors
  size_t plane;         // cells per plane (nx*ny*nz)
  double phifac;        // pending phidamp factor applied to the phi plane
  double faco, facn, fact;
  double gamma, gm1;
  int limiter;          // 0 flat, 1 minmod, 2 modified_mc
  int nvar;
  int tile[3];          // tile extent
  int tiles[3];         // tiles per axis
  int nspc;             // passive scalars (primitive planes NP.. of pin/pout)
  int stage;            // RK stage, 1-based
  double* spcorg;       // spc * density at stage 1 (rungekutta.f90:67), nspc planes
  // z slabs exchanging by push: the low ([0]) and high ([1]) neighbours'
  // halo buffers this stage's output layers go to (nullptr: no neighbour)
  double* push[2];
};

// Several whole steps of a small grid in one persistent launch
// (hmn_small.cu: small_run_kernel).
struct SmallRun {
  StageArgs st[2][3];   // [primitive buffer of the step's state][RK stage - 1]
  DevScalars* sc;
  unsigned int* bar;    // grid barrier: the arrival counter (zeroed before every launch)
  double phifac0;       // pending phidamp factor for the first step's stage 1
  double damp;          // the factor of every later step's stage 1 (1 without GLM)
  int nsteps, ntiles, rk;
};

// Arguments of one hyperbolic-gravity RK stage (hmn_kernels.cu: hg_stage_kernel).
struct HGArgs {
  const double* phi_in;
  const double* psi_in;
  double* phi_out;
  double* psi_out;
  double* org_phi;
  double* org_psi;
  const double* dens;  // density plane of the state at the gravity call
  size_t plane;
  double faco, facn, fdc;  // fdc = (fact*dtg)*cgrav
  double fourpiG;
  double damp;             // applied to psi after the last stage
  int stage1, last;
  DevScalars* sc;
  // spherical grids: the 8 coefficient planes of the Laplacian (c0, then the
  // -x, +x, -y, +y, -z, +z neighbours' weights, then the normalisation) and
  // the potential beyond r = xi1s as the last boundary pass left it
  const double* lc;
  const double* gin;
  // Cartesian grids uniform along every axis: the Laplacian weights every
  // cell would form (c0, the -/+ neighbour weights of each axis, the cell
  // volume cn) and RN(1/cn), formed once on the host with the same IEEE
  // operations; urcn_ok where cn lies in [2^-500, 2^501)
  int uni, urcn_ok;
  double uc0, ucm[3], ucp[3], ucn, urcn;
};

// One simulation of a batch, resident in device memory.  Every field the
// batched kernels need to run a step of this grid on its own clock.
struct SimDesc {
  GridDev G;
  double* U[3];       // conserved-state RK buffers (U^n in U[0])
  double* P[2];       // primitive planes, ping-pong
  size_t plane;
  int tiles[3];
  int pcur;           // P buffer of the current state
  int nvar, limiter, rktype, glm;
  int active;         // 0 for a free slot
  int held;           // 1: left out of the steps until released (hmn_batch_set_held)
  double gamma, gm1;
  double damp;        // phidamp factor exp(-alpha9wave*courant)
  double phifac;      // pending phidamp factor for the next stage 1
  DevScalars sc;      // this simulation's time, dt, ch, CFL reduction, errors
};

enum : int { kOK = 0, kEINVAL = -1, kENEG_EINT = -2, kECUDA = -3, kEBADCFG = -4, kENOMEM = -5, kETIMEOUT = -6 };

}  // namespace hmn

namespace hmn {
// launchers (hmn_kernels.cu)
void stage_tile(const int solve[3], int precision, int nspc, int tile[3], bool sph = false);
// tm: tensor maps of A.pin for TMA staging (3-D tiles; nullptr stages with plain loads)
cudaError_t launch_stage(const GridDev& G, const StageArgs& A, bool mag, bool glm, const TmaMaps* tm,
                         cudaStream_t st);
// the FP64 stage of a 3-D Cartesian grid without passive scalars as a march
// along z (hmn_march.cu); cudaErrorNotSupported for every other grid
cudaError_t launch_stage_march(const GridDev& G, const StageArgs& A, bool mag, bool glm, cudaStream_t st);
bool march_enabled();
// its decomposition: z planes per chunk, column tiles along x and y, chunks
void march_chunks(const int n[3], int* lz, int* ntx, int* nty, int* nch);
// up to R.nsteps steps of a small grid in one cooperative launch of at most
// one CTA per tile (hmn_small.cu); *grid receives the CTA count
int small_run_supported(const int tile[3], bool sph);
cudaError_t launch_small_run(const GridDev& G, const SmallRun& R, bool mag, bool glm, bool sph, const int tile[3],
                             cudaStream_t st, int* grid);
// mixed precision (hmn_mixed.cu): FP32 Riemann solver, FP64 reconstruction and accumulation
cudaError_t launch_stage_mixed(const GridDev& G, const StageArgs& A, bool mag, bool glm, const TmaMaps* tm,
                               cudaStream_t st);
// the two halves of launch_cfl: the per-cell reduction and the dt finalisation
cudaError_t launch_cfl_cells(const GridDev& G, const double* P, size_t plane, double gamma, DevScalars* sc,
                             bool mag, int nblocks, cudaStream_t st);
cudaError_t launch_cfl_finalize(DevScalars* sc, cudaStream_t st);
// the two boundary layers of each primitive plane next to the low / high z face
cudaError_t launch_pack_zhalos(const double* P, const int n[3], int nplanes, double* send_lo, double* send_hi,
                               int nblocks, cudaStream_t st);
cudaError_t launch_cfl(const GridDev& G, const double* P, size_t plane, double gamma, DevScalars* sc, bool mag,
                       int nblocks, cudaStream_t st);
cudaError_t launch_prim_init(double* P, size_t plane, bool mag, int nblocks, cudaStream_t st);
cudaError_t launch_prim_from_u(const double* U, double* P, size_t plane, bool mag, bool glm, int nblocks,
                               cudaStream_t st);
cudaError_t launch_prim_out(const double* P, size_t plane, double phifac, double gm1, double* out, double* p_out,
                            int nblocks, cudaStream_t st);
cudaError_t launch_hg_stage(const GridDev& G, const HGArgs& A, int nblocks, cudaStream_t st);
cudaError_t launch_hg_stage_sph(const GridDev& G, const HGArgs& A, cudaStream_t st);
cudaError_t launch_advance(DevScalars* sc, cudaStream_t st);
// evo_output totals: nblocks x kEvoQ partials in part, the kEvoQ sums in out
constexpr int kEvoQ = 10;
cudaError_t launch_evo(const GridDev& G, const double* P, size_t plane, const double* gphi, const double* sinc,
                       double* part, int nblocks, double* out, cudaStream_t st);
// batched launchers over a work list of (sim, tile) items; tile_kind selects
// the compile-time tile (see batch_tile_kind), grid = persistent CTAs; the
// stage launchers' queue is null for the static item split or a self-
// resetting {next item, CTAs finished} counter pair (hmn_queue.cuh)
int batch_tile_kind(const int solve[3]);
int batch_tile_variants(int kind, int* tile_ids);
void batch_tile_shape(int tile_id, int tile[3]);
cudaError_t launch_batch_cfl(SimDesc* sims, const int2* items, int nitems, int kind, bool mag, int grid,
                             cudaStream_t st);
cudaError_t launch_batch_finalize(SimDesc* sims, int nsims, cudaStream_t st);
cudaError_t launch_batch_stage(SimDesc* sims, const int2* items, int nitems, int kind, bool mag, bool glm,
                               int stage, int rk, int precision, int grid, int* queue, cudaStream_t st);
cudaError_t launch_batch_advance(SimDesc* sims, int nsims, cudaStream_t st);
int batch_stage_blocks_per_sm(int kind, bool mag, bool glm, int precision);
cudaError_t launch_batch_stage_mixed(SimDesc* sims, const int2* items, int nitems, int kind, bool mag, bool glm,
                                     int stage, int rk, int grid, int* queue, cudaStream_t st);
int batch_stage_mixed_blocks_per_sm(int kind, bool mag, bool glm);
}  // namespace hmn
