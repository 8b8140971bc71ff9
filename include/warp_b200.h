/*
 * warp_b200 C ABI: B200-native 3D electrostatic PIC step of WARP.
 *
 * Plain C types only (no torch, no C++). Every entry point returns 0 on
 * success or a negative WG_E* code; wg_last_error() gives the message. Grid
 * arrays use the reference's Fortran layout (x fastest):
 *   phi(-1:nx+1,-1:ny+1,-1:nz+1)   one guard cell (nxguardphi = 1)
 *   rho(0:nx,0:ny,0:nz)            no guard cell  (nxguardrho = 0)
 * Particle pointers are DEVICE pointers (SoA, float64); the Python layer
 * (warp_b200.fieldsolver / warp_b200.multigrid) moves host arrays in and out.
 * Work is queued on the context's stream (wg_set_stream); calls that return
 * host results synchronize that stream.
 *
 * Each entry point names the reference routine it replaces (paths relative
 * to the radiasoft/warp tree).
 */
#ifndef WARP_B200_H
#define WARP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WG_OK 0
#define WG_EINVAL (-1)       /* bad argument (shape, pointer, option) */
#define WG_ECUDA (-2)        /* CUDA runtime error */
#define WG_ESTATE (-3)       /* call out of order (e.g. solve before rho) */
#define WG_EOVERFLOW (-4)    /* fixed-point charge accumulator overflow */
#define WG_ENODEV (-5)       /* no CUDA device */
#define WG_ENOMEM (-6)       /* device allocation failed */
#define WG_ETOOLARGE (-7)    /* size beyond a fixed limit of the entry point */

typedef struct wg_ctx wg_ctx;

/* Mesh description (w3d.nx.., w3d.xmmin.., f3d.bounds; f3d.v:231-233). */
typedef struct {
  int nx, ny, nz;
  double xmmin, xmmax, ymmin, ymmax, zmmin, zmmax;
  int bounds[6]; /* 0 Dirichlet, 1 Neumann, 2 periodic: xlo,xhi,ylo,yhi,zlo,zhi */
} wg_grid;

/* Solver options (MultiGrid3D attributes, f3d.v:215-231). */
typedef struct {
  double mgparam;  /* SOR over-relaxation, default 1.2 */
  double mgtol;    /* tolerance; meaning set by tolkind */
  int mgmaxiters;  /* default 100 */
  int mgmaxlevels; /* default 101 */
  int downpasses;  /* default 1 */
  int uppasses;    /* default 1 */
  int lcndbndy;    /* subgrid conductor boundaries, default 1 */
  int precision;   /* 0: FP64 V-cycles (mgform=1 form of the reference)
                      1: FP32 V-cycles inside FP64 defect correction */
  int tolkind;     /* 0: mgerror = max|dphi| in volts (reference criterion)
                      1: relative residual max|rhs-A phi|/max|rhs| */
  int flags;       /* WG_SOLVE_* bits below */
  int mgmaxvcycles; /* > 0: full multigrid (fullmultigrid3dsolve,
                       f3d_mgrid.F:502-945; FullMultiGrid3D default 2): the
                       coarse levels, solved first from the restricted rho
                       with this many V-cycles each, give the starting phi
                       (the warm start is not used); 0: multigrid3dsolve */
} wg_solve_opts;

#define WG_SOLVE_GRAPH 1  /* replay each V-cycle from a captured CUDA graph */
#define WG_SOLVE_PDL 4    /* launch the solver's kernels with programmatic
                             dependent launch (each launch overlaps the end of
                             the previous kernel; same results) */

typedef struct {
  int mgiters;      /* V-cycles done */
  int converged;    /* 1 if the tolerance was met before mgmaxiters */
  double mgerror;   /* last max|dphi| (volts) */
  double relres;    /* last relative residual (when computed, else -1) */
} wg_solve_stats;

/* One particle species, device SoA arrays of length np (top.pgroup). A lost
 * particle has gaminv == 0 (stckxy3d convention, w3d.F:11520-11535). */
typedef struct {
  double *x, *y, *z, *ux, *uy, *uz, *gaminv;
  int64_t np;
  double q, m, w; /* charge, mass, macroparticle weight (sq, sm, sw) */
} wg_particles;

/* The same species stored in FP32 (28 bytes a particle instead of 56): the
 * particle arrays of the mixed-precision form, whose push runs in FP32. The
 * reference stores particles in FP64 only (top.pgroup); the _f32 entry
 * points below are its routines on this storage. q, m and w stay FP64. */
typedef struct {
  float *x, *y, *z, *ux, *uy, *uz, *gaminv;
  int64_t np;
  double q, m, w;
} wg_particles_f32;

/* Parameters of one particle advance (padvnc3d, w3d.F:1575). */
typedef struct {
  double dt;
  double prwall, prwallx, prwally; /* round absorbing aperture (top.prwall) */
  int use_lattice;                 /* apply the hard-edge quad tables */
  int center;                      /* WG_CENTER_* below; 0 = fullv */
} wg_push_params;

/* padvnc3d's `center` argument. During a run the velocities are half a step
 * ahead of the positions. Right after loading both are at t, so the first
 * step is HALFV and the steps after it FULLV; SYNCHV brings the velocities
 * back in step with the positions for diagnostics. */
#define WG_CENTER_FULLV 0  /* v t-dt/2 -> t+dt/2, x t -> t+dt (w3d.F:1862-1987) */
#define WG_CENTER_HALFV 1  /* v t -> t+dt/2, x t -> t+dt (w3d.F:1989-2125) */
#define WG_CENTER_SYNCHV 2 /* v t-dt/2 -> t, x unchanged (w3d.F:2187-2310) */

/* ---- context ----------------------------------------------------------- */

/* MultiGrid3D.__init__ + allocatedataarrays (scripts/multigrid.py:77,
 * scripts/fieldsolver.py:1622-1695): allocates every MG level on the current
 * CUDA device. */
int wg_create(const wg_grid* grid, wg_ctx** out);
int wg_destroy(wg_ctx* ctx);
/* Work is queued on this cudaStream_t (NULL = the legacy default stream). */
int wg_set_stream(wg_ctx* ctx, void* cuda_stream);
const char* wg_last_error(void);
/* getmglevels (f3d_mgrid.F:3654-3845): level sizes and cell sizes. */
int wg_level_info(wg_ctx* ctx, int* nlevels, int* dims, double* deltas, int maxlevels);
/* Device pointers of the solver's phi and rho (solver.phi / solver.rho,
 * Fortran layout above). */
int wg_arrays(wg_ctx* ctx, double** phi, double** rho);

/* ---- conductors (installconductor, scripts/multigrid.py:743-783) ---------- */

/* Adds a shape on every MG level via grid-line intercepts
 * (generateconductors.py:2750 getdatanew + f3d_conductors.F:12
 * conductordelfromintercepts). kind: 0 ZCylinderOut (generateconductors.py:3494),
 * 1 ZCylinder (:3305), 2 Sphere (:4009). dfill defaults to 2. */
int wg_conductors_add_shape(wg_ctx* ctx, int kind, double radius, double length, double voltage,
                            double xcent, double ycent, double zcent, int condid, double dfill);
/* Adds raw ConductorType points (f3d.v:105-164). kind 0: interior
 * (indx[3n], volt[n], ilevel[n]); kind 1: subgrid (indx[3n], dels[6n] in the
 * order mx,px,my,py,mz,pz, volt[6n], ilevel[n]). Host pointers. */
int wg_conductors_add_points(wg_ctx* ctx, int kind, int64_t n, const int32_t* indx, const double* dels,
                             const double* volt, const int32_t* ilevel);
/* checkconductors (f3d_mgrid.F:3964-4050): clip, dedupe, sort by level, and
 * upload to the device. */
int wg_conductors_finalize(wg_ctx* ctx);
int wg_conductors_clear(wg_ctx* ctx);
/* out[0] interior, out[1] even subgrid, out[2] odd subgrid point counts. */
int wg_conductors_counts(wg_ctx* ctx, int64_t* out);
/* Host copy of the finalized lists; which: 0 interior, 1 even, 2 odd. */
int wg_conductors_export(wg_ctx* ctx, int which, int32_t* indx, double* dels, double* volt, int32_t* ilevel);

/* ---- field solve ---------------------------------------------------------- */

/* multigrid3dsolve (f3d_mgrid.F:83-500), called through
 * MultiGrid3D.dosolve (scripts/multigrid.py:846-917). phi is the warm start
 * and the result; rho is left unchanged. */
int wg_solve(wg_ctx* ctx, const wg_solve_opts* opts, wg_solve_stats* stats);
/* Relative residual of the current phi (same definition as tolkind 1). */
int wg_relresidual(wg_ctx* ctx, double mgparam, double* out);
/* Residual field rhs - A phi of the current phi on the finest level, as in
 * residual3d (f3d_mgrid.F:3094-3598) with the conductor voltages imposed and
 * without the ppp scaling (the mgform = 2 correction right-hand side,
 * f3d_mgrid.F:340-358). out: device array in the rho layout; rhs = rho scaled
 * by mgparam/(2 eps0 (1/dx^2+1/dy^2+1/dz^2)), so out is in volts per SOR
 * update. Asynchronous on the context's stream. */
int wg_residual_field(wg_ctx* ctx, double mgparam, double* out);
/* getese3dfromrhophi (dw3d.F:708-777), no symmetry: the electrostatic energy
 * dx dy dz / 2 * sum(rho * phi) over the nodes 0..n of the current rho and phi,
 * summed in the reference's order (bit-identical). *out is a host double;
 * synchronizes the context's stream. */
int wg_field_energy(wg_ctx* ctx, double* out);

/* ---- particles -------------------------------------------------------------- */

/* setrho3d -> setrho3ddirect1 (w3d.F:7199, 7757-7960), via
 * MultiGrid3D.setsourcep (multigrid.py:492-511). Charge is accumulated in a
 * 64-bit fixed-point grid, so rho is bit-identical from run to run.
 * zero_first clears rho first (loadrho3d zeroes rho before depositing). */
int wg_deposit(wg_ctx* ctx, const wg_particles* p, int zero_first);
/* The deposit of wg_deposit in pieces, for a caller that streams particles
 * in (no counterpart in the reference; it replaces one wg_deposit of a
 * species whose arrays arrive chunk by chunk). wg_deposit_begin clears the
 * fixed-point accumulator; wg_deposit_add accumulates one piece (every piece
 * must carry the same q and w); wg_deposit_end converts into rho, replacing
 * it when zero_first is set. The result equals one wg_deposit of all pieces
 * bit for bit. None of the three synchronizes the stream: an accumulator
 * overflow is reported as WG_EOVERFLOW by the next wg_solve. wg_deposit
 * returns WG_ESTATE while a chunked deposit is open. */
int wg_deposit_begin(wg_ctx* ctx);
int wg_deposit_add(wg_ctx* ctx, const wg_particles* p);
int wg_deposit_end(wg_ctx* ctx, int zero_first);
/* The deposit of wg_deposit into a caller-owned rho(0:nx,0:ny,0:nz) array,
 * with no context and no allocation (no counterpart in the reference). For
 * callers that cannot let a library allocate device memory: host codes that
 * manage every device buffer themselves, or that keep a step free of
 * cudaMalloc/cudaFree because those synchronize the device. Its fixed-point
 * accumulator is a fixed array inside the library, so the grid is limited to
 * (nx+1)(ny+1)(nz+1) <= 1048576 nodes (8 MiB); larger grids get WG_ETOOLARGE.
 * Call with the device that holds rho and the particles current. The first
 * call on each device looks up that array's device address; make that first
 * call before any stream capture. Work is queued on `stream` (a
 * cudaStream_t, NULL = legacy default stream), which is synchronized before
 * return. Calls that overlap on one device (other streams or threads) share
 * the accumulator and race: serialize them. */
int wg_deposit_noalloc(const wg_grid* grid, const wg_particles* p, double* rho, int zero_first, void* stream);
/* applyrhoboundaryconditions3d (w3d.F:2660-2750) on rho. */
int wg_finalize_rho(wg_ctx* ctx);
/* sete3d -> sete_from_phi_linear3d (w3d.F:3656, 3963-4108), via
 * MultiGrid3D.fetchfieldfrompositions (multigrid.py:521-558). E is ADDED to
 * ex, ey, ez (device arrays). */
int wg_fetch_e(wg_ctx* ctx, const double* x, const double* y, const double* z, double* ex, double* ey,
               double* ez, int64_t np);
/* Hard-edge quadrupole tables per lattice cell, as set by setlattzt
 * (top_lattice.F:1852-2030) and read by applyquad (top_lattice.F:2985-3120).
 * Host arrays of length nzl+1. */
int wg_set_lattice(wg_ctx* ctx, const double* czs, const double* cze, const double* cdb, int nzl,
                   double zlmin, double dzl);
/* lcorrectede (f3d.v:152 Conductor3d.lcorrectede; used by
 * MultiGrid3D.fetchfieldfrompositions, scripts/multigrid.py:528-546): when
 * on, wg_fetch_e and wg_advance gather E with sete3dwithconductor, efetch = 1
 * (f3d_mgrid.F:4774-5220). Next to a conductor the field then comes from the
 * subgrid points' dels and volt (getefieldatconductorsubgrid, :4635-4735,
 * recomputed from the current phi at each call, over an icgrid built as
 * setupconductorfielddata, :4581-4632, does), and particles outside the grid
 * get no field. Off by default, as in the reference. */
int wg_set_correctede(wg_ctx* ctx, int on);
/* One fused step of padvnc3d (w3d.F:1575) followed by particleboundaries3d
 * (w3d.F:11292): gather E (sete_from_phi_linear3d), quad B (applyquad),
 * epush3d/bpush3d(ibpush=1)/epush3d/xpush3d (w3d.F:2752,2834,3070) as
 * prm->center selects, periz (top.F:4015) and the round-pipe absorber
 * (stckxy3d, w3d.F:11473). A SYNCHV step pushes no position and applies no
 * boundary. An unknown center is WG_EINVAL. */
int wg_advance(wg_ctx* ctx, const wg_particles* p, const wg_push_params* prm);
/* The FP32-storage forms of wg_deposit, wg_deposit_add and wg_advance
 * (setrho3d, padvnc3d; same citations). The deposit converts each position
 * to FP64 and accumulates the same 64-bit fixed-point weights, so rho differs
 * from the FP64 form only through the positions' FP32 rounding. The advance
 * gathers E in FP64 from the FP64 phi at the FP32 positions, then kicks,
 * rotates and drifts in FP32 (quads, periz and the pipe as wg_advance). */
int wg_deposit_f32(wg_ctx* ctx, const wg_particles_f32* p, int zero_first);
int wg_deposit_add_f32(wg_ctx* ctx, const wg_particles_f32* p);
int wg_advance_f32(wg_ctx* ctx, const wg_particles_f32* p, const wg_push_params* prm);
/* wg_advance followed by wg_deposit_add of the advanced particles, in one
 * pass over them (padvnc3d then setrho3d, w3d.F:1575 and 7757-7960, as
 * step3d orders them): the new positions are deposited from registers into
 * the open chunked deposit (wg_deposit_begin .. wg_deposit_end) with the same
 * fixed-point weights, so rho is bit-identical to the separate calls. No
 * reference counterpart as a single routine. WG_ESTATE without an open
 * deposit. */
int wg_advance_deposit(wg_ctx* ctx, const wg_particles* p, const wg_push_params* prm);
int wg_advance_deposit_f32(wg_ctx* ctx, const wg_particles_f32* p, const wg_push_params* prm);
/* getzmmnt global moments (top.F:521-1444): out[0] live count, 1 xbar,
 * 2 ybar, 3 xrms, 4 yrms, 5 epsx, 6 epsy (x' = ux/uz), 7 reserved. FP64,
 * deterministic order. */
int wg_moments(wg_ctx* ctx, const wg_particles* p, double* out);
/* The moment sums of getzmmnt, itask = 2 (top.F:814-860, 880-1160), for a
 * non-relativistic species with ifzmmnt = 2: zmmnts0[33] over all live
 * particles, and zmmnts[(nzmmnt+1)*33] (moment fastest) on the z grid of
 * nzmmnt cells over [zmmntmin, zmmntmax) relative to zbeam. Each particle is
 * extrapolated in time to the two planes around it, its velocity change
 * taken from uxo/uyo/uzo (device arrays of the velocities dt earlier; the
 * reference calls this in the synchv step with the pre-synchv velocities
 * and dt = dt/2), and added to both with its linear weights times dtscale;
 * the extrapolation time is clipped at zmmntdtextmax*dt. The moment index k
 * is the reference's k+1. Sums are FP64 with atomic accumulation: they match
 * the serial sums to rounding, not bit for bit. Output arrays are host
 * memory; synchronizes the stream. */
int wg_zmoments(wg_ctx* ctx, const wg_particles* p, const double* uxo, const double* uyo, const double* uzo,
                double dt, double dtscale, double zbeam, double zmmntmin, double zmmntmax, int nzmmnt,
                double zmmntdtextmax, double* zmmnts0, double* zmmnts);

/* wg_moments and wg_zmoments for FP32 storage (uxo/uyo/uzo are FP32 device
 * arrays); the sums are FP64. */
int wg_moments_f32(wg_ctx* ctx, const wg_particles_f32* p, double* out);
int wg_zmoments_f32(wg_ctx* ctx, const wg_particles_f32* p, const float* uxo, const float* uyo, const float* uzo,
                    double dt, double dtscale, double zbeam, double zmmntmin, double zmmntmax, int nzmmnt,
                    double zmmntdtextmax, double* zmmnts0, double* zmmnts);

/* Cell keys for sorting particles by cell, as particlesortxyzwithcopy
 * (top.F:5095-5130): key = ix + (nx+1)*(iy + (ny+1)*iz); lost particles get
 * (nx+1)(ny+1)(nz+1). keys: device int64 array of length np. */
int wg_particle_keys(wg_ctx* ctx, const wg_particles* p, int64_t* keys);
/* Gathers dst[i] = src[perm[i]] for the 7 particle arrays (device perm of
 * length np; src and dst must not overlap). With perm from a stable sort of
 * the keys this is particlesortbyindex (top.F:5132). */
int wg_particle_permute(wg_ctx* ctx, const int64_t* perm, const wg_particles* src, const wg_particles* dst);
/* The same two for FP32 storage (particlesortxyzwithcopy, top.F:5095-5132). */
int wg_particle_keys_f32(wg_ctx* ctx, const wg_particles_f32* p, int64_t* keys);
int wg_particle_permute_f32(wg_ctx* ctx, const int64_t* perm, const wg_particles_f32* src,
                            const wg_particles_f32* dst);

/* ---- instrumentation (no reference counterpart: replaces the wall-clock
 * sub-timers lf3dtimesubs / lw3dtimesubs, f3d.v:1308, w3d.v:1396) -------- */

#define WG_PROF_SOR0 0     /* SOR half pass on the finest level, k_sor_bulk launches (units: nodes) */
#define WG_PROF_DEPOSIT 1  /* charge deposition (units: particles) */
#define WG_PROF_ADVANCE 2  /* fused gather + push (units: particles) */
#define WG_PROF_RESID0 3   /* residual on the finest level (units: nodes) */
#define WG_PROF_RESTRICT0 4 /* restriction from the finest level (units: fine nodes) */
#define WG_PROF_EXPAND0 5   /* prolongation into the finest level (units: fine nodes) */
#define WG_PROF_CORR 6      /* FP64 correction update of the mixed form (units: nodes) */
#define WG_PROF_COARSE 7    /* all work below the finest level in one V-cycle (units: level-1 nodes);
                               timed as a replay of its own captured graph with
                               the solve's PDL setting, as it runs in a V-cycle */

/* Starts CUDA-event timing of the kernel kinds in `mask` (bits 1<<WG_PROF_*),
 * clearing earlier records; mask 0 stops it. */
int wg_prof_enable(wg_ctx* ctx, int mask);
/* Sums the device time (ms), launch count and algorithmic units of one
 * kind recorded since wg_prof_enable. Synchronizes the stream. */
int wg_prof_read(wg_ctx* ctx, int kind, double* total_ms, int64_t* launches, double* units);
/* Number of kernels this context has launched since it was created. */
int wg_launch_count(wg_ctx* ctx, int64_t* n);

/* ---- learned warm start: BF16 tensor-core 3x3x3 convolutions (no
 * reference counterpart: WARP has no learned components) ------------------ */

/* y[v][yoff+co] = relu?(bias[co] + sum_{t,ci} x[v+off_t][ci] * W[t][co][ci]),
 * optionally multiplied by (mask[v][co] > 0). x: [D][H][W][cin] bf16; w: the
 * weights W packed as [27][cin/8][cout][8] bf16, i.e. w[t][g][co][j] =
 * W[t][co][8g+j] (tap t = 9*(dz+1) + 3*(dy+1) + (dx+1)); bias fp32 or NULL;
 * y: [D][H][W][ystride] bf16. cin, cout multiples of 16, cout <= 256; x, w, y
 * 16-byte aligned. Zero padding outside the box. *err is set non-zero if a
 * wait timed out. */
int wg_conv3_fwd(const void* x, int D, int H, int W, int cin, const void* w, const float* bias, int cout, void* y,
                 int ystride, int yoff, const void* mask, int mstride, int relu, int* err, void* stream);
/* wg_conv3_fwd with y in FP32 ([D][H][W][ystride] float, ystride and yoff
 * multiples of 4): the accumulator, bias, ReLU and mask without the rounding
 * to bf16. The last layer of the learned guess writes this, so that the
 * correction added to phi carries no bf16 rounding noise. */
int wg_conv3_fwd_f32(const void* x, int D, int H, int W, int cin, const void* w, const float* bias, int cout,
                     float* y, int ystride, int yoff, const void* mask, int mstride, int relu, int* err,
                     void* stream);
/* dw[t][co][ci] = sum_v dy[v][co] * x[v+off_t][ci] (fp32; overwritten), from
 * x: [D][H][W][cin] and dy: [D][H][W][cout] bf16 (16-byte aligned), cin a
 * multiple of 16 up to 256, cout a multiple of 16 up to 128. CTAs write
 * partial sums to `scratch` (device, at least the size wg_conv3_wgrad_scratch
 * reports) and a second kernel adds them in a fixed order: the result is the
 * same bits on every run. *err is set non-zero if a wait timed out. */
int wg_conv3_wgrad(const void* x, const void* dy, int D, int H, int W, int cin, int cout, float* dw, float* scratch,
                   int64_t scratch_floats, int* err, void* stream);
/* Floats of scratch wg_conv3_wgrad needs for (cin, cout) on the current device. */
int wg_conv3_wgrad_scratch(int cin, int cout, int64_t* nfloats);

#ifdef __cplusplus
}
#endif

#endif /* WARP_B200_H */
