/* vh.h - C ABI of the B200 viscous Kurganov-Tadmor hydro step.
 *
 * Drop-in boundary for the CPU step of rjfries/VIRAL ("3-1ViscousHydro").
 * The reference has no library API: its step is TVDRK2(GRID, tau, ts)
 * operating on a global grid (NEWEST5/time.h:333), initialised by
 * init(tau, ts) (NEWEST5/init.h:556), stopped by MaxTempGev (NEWEST5/
 * utils.h:263) and written by WriteResults[XY] (NEWEST5/write.h:51,225).
 * This header replaces those entry points with a handle-based interface:
 * no globals, no exit(), plain pointers and sizes, an int status on every
 * call.  Every entry point cites the reference routine it stands in for.
 *
 * State layout (host and device): structure of arrays over the
 * ghost-inclusive grid GX x GY x GZ with GX = nx + 6, GY = ny + 6,
 * GZ = nz + 6 (or 1 when boost invariant), index (k*GY + j)*GX + i, x
 * fastest; 3 ghost layers per face as the reference's BORDER
 * (NEWEST5/maindef.h:369-371).  The 18 state fields, in this order:
 *   0 e, 1..4 u^tau u^x u^y u^eta, 5..9 pi^xx pi^yy pi^xy pi^x-eta pi^y-eta,
 *   10..13 T^{tau tau} T^{tau x} T^{tau y} T^{tau eta}, 14..17 previous u^mu
 * (the reference's cell fields En, u[4], pi[5], T00..T30, prevu[4],
 * NEWEST5/maindef.h:392-466).  Units: fm^-4 for e, pi and T^{mu nu},
 * fm^-1 for temperature, fm for lengths, fm/c for tau.
 *
 * Threading: one handle per host thread; calls on a handle are issued on
 * that handle's CUDA stream (vh_set_stream) and do not synchronise except
 * where a result is returned to the host.
 */
#ifndef VH_H
#define VH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VH_NFIELDS 18
#define VH_NGHOST 3

typedef enum {
  VH_OK = 0,
  VH_E_ARG = 1,        /* bad argument (null pointer, size, enum) */
  VH_E_CUDA = 2,       /* a CUDA call failed; see vh_last_error */
  VH_E_ROOTFIND = 3,   /* conserved-to-primitive Newton failed in some cell
                          (NEWEST5/multiroot.h:398-420 exits there) */
  VH_E_CAUSALITY = 4,  /* |v| >= 1 after the root-find (multiroot.h:480-488) */
  VH_E_NEG_ENERGY = 5, /* e <= 0 after the root-find (multiroot.h:480-488) */
  VH_E_TIMEOUT = 6,    /* a bounded device wait ran out */
  VH_E_STATE = 7,      /* call out of order (e.g. step before state is set) */
  VH_E_NOMEM = 8,      /* device allocation failed */
  VH_E_UNSUPPORTED = 9 /* option not built into this library */
} vh_status;

enum { VH_COORD_MILNE = 0, VH_COORD_CARTESIAN = 1 };
enum { VH_PREC_FP64 = 0, VH_PREC_MIXED = 1 };
enum { VH_RECON_WENO5 = 0, VH_RECON_MINMOD = 1 };
enum { VH_EOS_CONFORMAL = 0, VH_EOS_TABLE = 1 };
/* relaxation time: 1.5 eta / P (NEWEST5/maindef.h:69,126,286) or
 * 5 eta / (e + P) (NEWEST5/maindef.h:339, the Gubser test) */
enum { VH_TAUPI_15_ETA_OVER_P = 0, VH_TAUPI_5_ETA_OVER_EPP = 1, VH_TAUPI_CONST = 2 };
/* initial pi: given, zero, or Navier-Stokes (NEWEST5/Source.h:535-630) */
enum { VH_PI_GIVEN = 0, VH_PI_ZERO = 1, VH_PI_NS = 2 };
/* snapshot layouts: NEWEST5/write.h's 12 doubles per cell for one xy plane
 * or the full grid, and NEWEST10/write.h's 17 (full pi^{mu nu}) likewise */
enum { VH_WRITE_XY = 0, VH_WRITE_FULL = 1, VH_WRITE_XY17 = 2, VH_WRITE_FULL17 = 3, VH_WRITE_NS_XY = 4 };

typedef struct {
  int coords;           /* VH_COORD_* (NEWEST5 Milne, TXYZ5 Cartesian) */
  int precision;        /* VH_PREC_FP64, or VH_PREC_MIXED: FP32 state, fluxes,
                           reconstruction and sources; FP64 root-find, EOS
                           inversion and compensated conservation sums.
                           Range of the mixed mode: its WENO5 weights take
                           one FP32 division per face pair, whose divisor
                           grows as the eighth power of the stencil's
                           differences; differences of a reconstructed
                           quantity (tau T^{tau mu}, pi^{mu nu}, the fluxes,
                           u^mu) above about 1e4 in fm units (e.g. energy-
                           density spikes above about 2000 GeV/fm^3 across a
                           cell) overflow it.  Run such states in FP64. */
  int recon;            /* VH_RECON_* */
  int nx, ny, nz;       /* interior cells (nz = 1 when boost_invariant) */
  int boost_invariant;  /* 1: no eta direction, no eta ghosts (reference LBI) */
  double dx, dy, dz;    /* cell sizes (fm, fm, 1 or fm) */
  double tau0, dtau;    /* start time and step (fm/c) */
  int eos_kind;         /* VH_EOS_* */
  double eos_a;         /* conformal EOS: e = a T^4 in fm units */
  int eos_n;            /* table rows (log-spaced in e, increasing) */
  const double* eos_e;  /* table: e (fm^-4) */
  const double* eos_p;  /* table: P (fm^-4) */
  const double* eos_cs2;/* table: dP/de */
  const double* eos_t;  /* table: T (fm^-1) */
  /* eta/s(T) = etas0 + etas1 * max(T*hbarc - etas_tc, 0), T*hbarc in GeV */
  double etas0, etas1, etas_tc, hbarc;
  int taupi_kind;       /* VH_TAUPI_* */
  int gubser_mirror;    /* ghost u^x,u^y mirrored across the face (NEWEST5/
                           boundary.h:32-37, Gubser test) */
  double minmod_theta;  /* generalized-minmod theta (NEWEST5/maindef.h:370) */
  double taupi_const;   /* VH_TAUPI_CONST: tau_pi in fm/c (the Bjorken block,
                           NEWEST5/maindef.h:228) */
  int cold_plasma;      /* 1: the shear source without its relaxation term
                           -pi/tau_pi (the reference's COLDPLASMA test of the
                           Gubser flow, NEWEST5/Source.h:371-410) */
} vh_config;

typedef struct vh_handle vh_handle;

/* Create a handle and allocate the device state for one event.
 * Replaces StoreInHeap/init bookkeeping (NEWEST5/alloc.h:33, init.h:556-589). */
int vh_create(const vh_config* cfg, vh_handle** out);
/* Free everything (NEWEST5/alloc.h FreeFromHeap). */
int vh_destroy(vh_handle* h);
/* Issue all later work on this cudaStream_t (NULL: the legacy stream). */
int vh_set_stream(vh_handle* h, void* stream);
/* Extents of the ghost-inclusive grid. */
int vh_dims(const vh_handle* h, int* gx, int* gy, int* gz);

/* Full state from / to host memory, 18 fields x GX*GY*GZ doubles.
 * Setting the state sets the current time to tau. */
int vh_set_state(vh_handle* h, const double* host, double tau);
int vh_get_state(vh_handle* h, double* host);
/* The same with device pointers to 18 x G doubles (no host copies). */
int vh_set_state_device(vh_handle* h, const double* dev, double tau);
int vh_get_state_device(vh_handle* h, double* dev);
/* Primitive fields of every ghost-inclusive cell, as the reference's cell
 * holds them (NEWEST5/maindef.h:392-466: En, P, Temp, u[4], and pi with its
 * dependent components A1..A5, maindef.h:497-501): e, P, T (n doubles each),
 * u^mu (4 x n) and pi^{mu nu} (10 x n, contravariant, in the order tt, tx,
 * ty, t-eta, xx, xy, x-eta, yy, y-eta, eta-eta), in fm units.  Any pointer
 * may be NULL. */
int vh_get_primitive(vh_handle* h, double* e, double* P, double* T, double* u4, double* pi10);

/* Landau matching (NEWEST5/ginit.h:521-656, FindVar): for each of n cells
 * the timelike eigenvector u^mu (u_mu u^mu = 1) of T^mu_nu and its
 * eigenvalue e, from the contravariant T^{mu nu} given as 10 x n doubles
 * (tt, tx, ty, t-eta, xx, xy, x-eta, yy, y-eta, eta-eta) at time tau (Milne
 * metric diag(1,-1,-1,-tau^2); Cartesian when cartesian != 0).  Outputs e
 * (n) and u (4 x n); *nfail (may be NULL) counts the cells without a
 * timelike eigenpair (where the reference exits).  Runs on the current GPU;
 * the arrays are host memory. */
int vh_landau_match(const double* tmunu10, long long n, double tau, int cartesian, double* e, double* u4,
                    long long* nfail);
/* Initial state from T^{mu nu} on the handle's ghost-inclusive grid (10 x n
 * host doubles as above), as the reference's Glasma initialisation builds it
 * (NEWEST5/ginit.h:658-1052): Landau matching, P(e) from the EOS, and the
 * five evolved components of pi^{mu nu} = T^{mu nu} - T_id^{mu nu}
 * - PI (g^{mu nu} - u^mu u^nu), T_id = (e+P) u u - P g, PI = -(e - 3P)/3
 * (the trace of T_id: for the traceless field tensor pi comes out
 * traceless; PI is not evolved), prevu = u, T^{tau mu} from (e, u, pi).
 * VH_E_ROOTFIND, with *nfail > 0, when some cell has no timelike eigenpair. */
int vh_init_tmunu(vh_handle* h, double tau, const double* tmunu10, long long* nfail);
/* prevu from T^{mu nu} at tau_prev = tau0 - dtau by Landau matching, after
 * vh_init_tmunu (the reference calls ginit at tau0 - ts first and keeps
 * only the velocity, NEWEST5/init.h:658-662, ginit.h:945-953). */
int vh_init_prevu_tmunu(vh_handle* h, double tau_prev, const double* tmunu10, long long* nfail);
/* The reference's optical-Glauber CGC tensor (NEWEST5/ginit.h:658-913) at
 * tau on the ghost-inclusive grid of nx x ny (x nz) cells: T^{mu nu} in the
 * order of vh_landau_match.  Thickness functions mu1, mu2 of two
 * Woods-Saxon nuclei (mass number, diffuseness ws_a; R = 1.12 A^(1/3) -
 * 0.86 A^(-1/3)) centred at x = +x_pos and -x_pos, integrated along the
 * beam axis and scaled by 2 thickness_scale; e = N mu1 mu2 with N setting
 * the grid maximum to e_peak (fm^-4; the reference uses 0.58 e_max(tau),
 * e_max from T = 0.4 GeV at 0.6 fm/c scaled by (tau/0.6)^(-4/3));
 * alpha = -grad e, beta = N (mu1 grad mu2 - mu2 grad mu1) by WENO
 * derivatives (of log mu for the thicknesses); T^{mu nu} to order tau^2
 * with the coefficient delta (the reference's 100) of its e-proportional
 * terms; an eta profile flat for |eta| < eta_flat/2 with unit-width
 * Gaussian tails.  The reference's values: x_pos 3, A 197, ws_a 0.546,
 * thickness_scale 12.2546, eta_flat 4, delta 100.  Host arrays. */
int vh_profile_cgc(int nx, int ny, int nz, int boost_invariant, double dx, double dy, double dz, double tau,
                   double x_pos, double mass_number, double ws_a, double thickness_scale, double e_peak,
                   double eta_flat, double delta, double* tmunu10);

/* Initialise from a profile (the reference's init(tau, ts) with a scenario,
 * NEWEST5/init.h:556-704): e, u^x, u^y, u^eta on the ghost-inclusive grid
 * (u^tau from normalisation), optional previous velocity prevu (4 fields;
 * NULL: prevu = u), and pi by pi_mode: VH_PI_GIVEN takes pi5 (5 fields),
 * VH_PI_ZERO sets 0, VH_PI_NS computes Navier-Stokes pi on every cell
 * (NEWEST5/Source.h:607-630).  T^{tau mu} follows from (e,u,pi)
 * (NEWEST5/init.h:539-549).  Host arrays of G doubles each. */
int vh_init_profile(vh_handle* h, double tau, const double* e, const double* ux, const double* uy,
                    const double* ueta, const double* prevu4, int pi_mode, const double* pi5);

/* Advance nsteps TVDRK2 steps of dtau (NEWEST5/time.h:333 TVDRK2, called
 * from the main loop NEWEST5/main.cpp:132-206).  Returns VH_E_ROOTFIND /
 * VH_E_CAUSALITY / VH_E_NEG_ENERGY if a cell failed (the state is then
 * that of the failing step). */
int vh_step(vh_handle* h, int nsteps);
/* Current time tau. */
int vh_get_time(const vh_handle* h, double* tau);

/* Maximum temperature over the interior in GeV (NEWEST5/utils.h:263). */
int vh_max_temperature(vh_handle* h, double* tmax_gev);
/* Compensated FP64 sums over the interior of tau*T^{tau mu} times the cell
 * volume: out[4] = {E, Px, Py, Peta} (conservation monitor). */
int vh_conservation_sums(vh_handle* h, double* out4);
/* Largest signal speed over the interior faces and the CFL step
 * dx/(8 max|lambda|) the reference suggests (NEWEST5/hydroKT.h:317-344). */
int vh_cfl(vh_handle* h, double* max_speed, double* dtau_suggest);

/* Snapshot in the reference's binary layout: 12 doubles per interior cell
 * (e, T, P, v^x, v^y, v^eta, pi^xx..pi^y-eta, Pi), x outer, y inner, at
 * the central eta slice (VH_WRITE_XY, NEWEST5/write.h:51-115) or for every
 * eta slice (VH_WRITE_FULL, NEWEST5/write.h:225-290); `every` keeps every
 * n-th cell as the reference's FREQ. */
int vh_write(vh_handle* h, const char* path, int layout, int every);
/* VH_WRITE_XY17 / VH_WRITE_FULL17: the same two layouts with 17 doubles per
 * cell (e, T, P, v^x, v^y, v^eta, the ten pi^{mu nu} in the order tt, tx, ty,
 * t-eta, xx, xy, x-eta, yy, y-eta, eta-eta, Pi), NEWEST10/write.h:51-115 and
 * its WriteResults. */

/* The reference's evolved variables Var[10] on every cell (CopyPrimary-
 * VariablesToVar, NEWEST5/hydroKT.h:345-361): tau T^{tau mu} (T^{t mu} in
 * Cartesian coordinates, TXYZ5/hydroKT.h:270-286), pi^{xx}, pi^{yy},
 * pi^{xy}, pi^{x eta}, pi^{y eta}, and the bulk pressure (zero): 10 fields
 * of the ghost-inclusive grid. */
int vh_get_conserved(vh_handle* h, double* var10);

/* VH_WRITE_NS_XY: NEWEST10's Navier-Stokes snapshot (WriteNSXY,
 * NEWEST10/write.h:123-170, written as res/NStau%2.3ffm.bin): 11 doubles
 * per cell, the ten components of vh_get_ns_pi and a zero bulk part, in the
 * VH_WRITE_XY order (x outer, y inner, central eta slice, every FREQ-th). */

/* Navier-Stokes shear pi^{mu nu}_NS = 2 eta sigma^{mu nu} at the current
 * state, ten fields of the ghost-inclusive grid in the order tt, tx, ty,
 * t-eta, xx, xy, x-eta, yy, y-eta, eta-eta (NEWEST10/Source.h:643-753,
 * CalcNS), with the step's velocity derivatives: d_tau u = (u - prevu)/dtau
 * and WENO derivatives in space (NEWEST10/Source.h:3-95).  Meaningful on
 * the interior cells.  Evaluated in FP64 (from the FP32 state in the mixed
 * mode). */
int vh_get_ns_pi(vh_handle* h, double* pi10);

/* Restart files.  vh_save_checkpoint writes the grid, tau and the 18
 * canonical fields of every cell (ghosts and the previous velocity
 * included); vh_load_checkpoint restores them into a handle of the same grid
 * (coordinates, nx, ny, nz, boost invariance, dx, dy, dz; VH_E_ARG
 * otherwise) and sets *tau_out (may be NULL).  A run resumed from a file of
 * its own precision continues bit for bit; the handle's dtau applies.  The
 * reference has no restart state (its snapshots are output only). */
int vh_save_checkpoint(vh_handle* h, const char* path);
int vh_load_checkpoint(vh_handle* h, const char* path, double* tau_out);

/* Initial profile from the ASCII files of the ideal-hydro driver
 * (NEWideal/init.h:296-345): eps_path, vx_path and vy_path hold nx*ny
 * whitespace-separated numbers each, x fastest, for the interior cells of a
 * boost-invariant grid.  Writes e, u^x, u^y on the ghost-inclusive grid
 * ((nx+6)*(ny+6) doubles each; u = v / sqrt(1 - v^2)) with the reference's
 * floor: every cell below 0.01 (the ghost cells included) gets min/10, min
 * being the smallest interior value above 1e-5 in magnitude (100 if none is
 * smaller); *min_out receives it (may be NULL).  VH_E_ARG when a file cannot
 * be read or holds fewer than nx*ny numbers. */
int vh_read_ideal_profile(const char* eps_path, const char* vx_path, const char* vy_path, int nx, int ny,
                          double* e, double* ux, double* uy, double* min_out);

/* Stage-1 terms for tests: the flux divergence res[9*G], sources src[9*G]
 * and velocity gradients du[16*G] at the current state (the reference's
 * CalcSource + hydroExplicit, NEWEST5/Source.h:165, hydroKT.h:391). */
int vh_debug_stage_terms(vh_handle* h, double* res, double* src, double* du);

/* Diagnostic: advance nsteps steps with a CUDA event pair around every
 * kernel launch and return device milliseconds summed per kernel kind:
 * ms_out[0..2] the x / y / eta flux kernels, ms_out[3] the stage-1 update,
 * ms_out[4] the stage-2 update.  Slower than vh_step (one sync per launch). */
int vh_time_kernels(vh_handle* h, int nsteps, double* ms_out);

/* Newton iterations of the last step, summed over cells (diagnostic). */
int vh_last_iterations(vh_handle* h, long long* iters);

/* How the flux sweeps read their tiles (diagnostic): *tma = 1 when each
 * tile is staged in shared memory by tensor-memory-accelerator box copies
 * (cp.async.bulk.tensor from tensor maps over the state), 0 when the
 * threads load it through the cache.  TMA is the default; VH_TMA=0 in the
 * environment at vh_create selects the cached loads (same arithmetic). */
int vh_sweep_uses_tma(const vh_handle* h, int* tma);

/* Step without allocating: the FP64 step of vh_step on device memory the
 * caller owns, for callers that must not call cudaMalloc where they step the
 * fluid (a device memory pool owned by another framework, whose budget a
 * cudaMalloc behind its back would break).  No counterpart in the reference,
 * which steps host memory it allocated itself.
 *   state:   device pointer to the 18 canonical fields (18 x G doubles),
 *            read and advanced in place by nsteps steps from tau
 *   eos_dev: device copy of the EOS table [e | P | cs2 | T] (4 x eos_n
 *            doubles) when cfg->eos_kind is VH_EOS_TABLE, else NULL;
 *            cfg->eos_e must still point to the host table (positive and
 *            strictly increasing)
 *   stream:  cudaStream_t to launch on (NULL: the legacy stream)
 * cfg->precision must be VH_PREC_FP64, cfg->taupi_kind one of the two
 * eta-proportional forms, cfg->cold_plasma 0, tau > 0 on Milne grids, and the
 * ghost-inclusive grid at most VH_STATIC_MAX_CELLS cells, else VH_E_ARG.  The
 * step's scratch is one file-scope device array of 16 MiB that every GPU
 * loading the library holds until exit; all calls share it and it keeps the
 * last call's contents, so calls that overlap on the GPU race (issue them one
 * after another).  The first call on a device looks up that array's address.
 * Each call copies its status word to the host and synchronises stream before
 * it returns; the return codes are vh_step's. */
#define VH_STATIC_MAX_CELLS 61680
int vh_step_static(const vh_config* cfg, double* state, const double* eos_dev, double tau, int nsteps,
                   void* stream);

/* ------------------------------------------------------------- batches */
/* An ensemble of boost-invariant Milne events evolved together by one
 * persistent kernel over a packed event table (one device pool for all
 * events).  Every event has its own grid (nx[i] x ny[i]), start time, step
 * and maximum time; it stops when its maximum temperature falls below
 * t_freeze_gev or its time reaches tau_max (the reference's main-loop
 * breaks, NEWEST5/main.cpp:188-205, applied per event), or fails alone
 * (root-find / causality) while the others continue.  The common physics
 * (EOS, transport, precision, reconstruction, dx, dy) comes from cfg; its
 * grid and time fields are ignored. */
typedef struct vh_batch vh_batch;
enum { VH_EVENT_RUNNING = 0, VH_EVENT_FROZEN = 1, VH_EVENT_TAUMAX = 2, VH_EVENT_FAILED = 3 };
int vh_batch_create(const vh_config* cfg, int n_events, const int* nx, const int* ny, const double* tau0,
                    const double* dtau, const double* tau_max, double t_freeze_gev, vh_batch** out);
int vh_batch_destroy(vh_batch* b);
/* rewind every event to its start time and running state (the pool keeps
 * its contents; re-initialise the events to restart them) */
int vh_batch_reset(vh_batch* b);
/* one event's initial profile on its ghost-inclusive grid (as vh_init_profile) */
int vh_batch_init_event(vh_batch* b, int ev, const double* e, const double* ux, const double* uy,
                        const double* prevu4, int pi_mode, const double* pi5);
/* every event from the MC-Glauber generator (vh_profile_glauber with the
 * event's seed and impact parameter), u = 0, pi = 0; host threads */
int vh_batch_init_glauber(vh_batch* b, const uint64_t* seeds, const double* bimp, int A, double R, double aws,
                          double dmin, double sigma_nn, double w, double epeak_gev, double efloor_gev,
                          int nthreads, int* npart_out);
/* run until every event has stopped or max_steps steps; device seconds and
 * whether the launches were replayed from a CUDA graph */
int vh_batch_run(vh_batch* b, int max_steps, double* seconds, int* graph_used);
/* per-event time, steps taken and state (VH_EVENT_*) */
int vh_batch_events(vh_batch* b, double* tau, int* steps, int* state);
/* one event's 18 canonical fields (doubles, its ghost-inclusive grid) */
int vh_batch_get_event_state(vh_batch* b, int ev, double* host18);
/* pick the persistent kernel's tile shape (lines per tile), occupancy,
 * flux-loop unroll and steps per launch by timing probe_steps steps of each
 * candidate; cached by device, precision and event-size histogram in
 * cache_path (NULL: no cache) */
int vh_batch_autotune(vh_batch* b, const char* cache_path, int probe_steps, double* best_ms_per_step);
int vh_batch_set_tuning(vh_batch* b, int variant, int steps_per_launch, int use_graph);
int vh_batch_get_tuning(vh_batch* b, int* variant, int* steps_per_launch, int* lines_per_tile, int* blocks_per_sm,
                        int* unroll);
/* Per-event observables of the events' current states (no counterpart in
 * the reference, which only evolves): the momentum anisotropy eps_p (as
 * vh_eps_p) and the eccentricity of the energy density about its centre,
 * eps_2 = sqrt((<y^2> - <x^2>)^2 + 4 <xy>^2) / (<x^2> + <y^2>); n doubles
 * each, either may be NULL. */
int vh_batch_observables(vh_batch* b, double* eps_p, double* ecc2);
/* Self-test of the bounded grid barrier of the persistent kernel: a launch of
 * two blocks where absent_blocks (0 or 1) never arrive.  With one absent, the
 * waiting block gives up after its spin limit (2^20 polls) and the call
 * returns VH_E_TIMEOUT, as vh_batch_run does when a barrier times out; the
 * context stays usable.  *seconds (may be NULL) receives the launch's time. */
int vh_batch_barrier_selftest(int absent_blocks, double* seconds);
const char* vh_batch_last_error(const vh_batch* b);

/* ------------------------------------------------------------- adjoint
 * Gradients of a final-time flow observable (no counterpart in the
 * reference, whose driver only evolves; NEWEST5/time.h:333 is the step that
 * is differentiated). */

/* Momentum anisotropy of the current state, summed in FP64 over the interior
 * cells: eps_p = sum(T^xx - T^yy) / sum(T^xx + T^yy), with
 * T^ij = (e + P) u^i u^j + P delta^ij + pi^ij.  Milne grids, summed over
 * every interior cell (every eta slice of a 3+1D grid). */
int vh_eps_p(vh_handle* h, double* eps_p);

/* Discrete adjoint of eps_p after nsteps steps from the current state
 * (Milne grids, boost-invariant or 3+1D, WENO reconstruction, copy
 * boundaries; VH_E_UNSUPPORTED otherwise).  Runs
 * the forward in segments of checkpoint_every steps (the first segment takes
 * the remainder), checkpointing the state at each segment start, then the
 * reverse of every step, re-running each segment from its checkpoint (the
 * last one is recorded during the forward).  The
 * max-speed and limiter branches are the forward pass's; the root-find is
 * differentiated through the implicit-function theorem.  Outputs (each may
 * be NULL):
 *   eps_p       the observable at the final time;
 *   grad_state  18 x n doubles, canonical field order: d eps_p / d (initial
 *               state), every field an independent variable (fields the step
 *               never reads get 0);
 *   grad_e      n doubles: d eps_p / d e of vh_init_profile, i.e. with
 *               T^{tau mu} = (e + P) u^tau u^mu - P g^{tau mu} + pi^{tau mu}
 *               re-derived from e at fixed u and pi (ghost cells included);
 *   grad_etas   2 doubles: d eps_p / d (etas0, etas1) of vh_config.
 * The handle is left at the final state.  In the mixed mode the adjoint runs
 * in FP32 with the implicit-function solve in FP64. */
int vh_adjoint_eps_p(vh_handle* h, int nsteps, int checkpoint_every, double* eps_p, double* grad_state,
                     double* grad_e, double* grad_etas);
/* Device milliseconds of the last vh_adjoint_eps_p on this handle: [0] the
 * forward with its checkpoints, [1] the recomputation of the segments with
 * their records, [2] the reverse steps, [3] the rest (seed, gradient export,
 * state restore, and the workspace allocation of a first call). */
int vh_adjoint_phase_times(const vh_handle* h, double* ms4);

/* Message of the last error on this handle (or the last vh_create). */
const char* vh_last_error(const vh_handle* h);

/* ---------------------------------------------------------------- inputs */
/* Seeded host generators shared by the GPU path and its tests, so that
 * identical inputs hold by construction.  All fill ghost-inclusive arrays. */

/* Synthetic tabulated EOS: n rows log-spaced in e over [emin, emax] GeV/fm^3,
 * c_s^2(e) = 1/3 - 0.2 exp(-ln^2(e/0.5)/2), P(emin) = c_s^2(emin) emin,
 * T anchored to e = a T^4 at emax; outputs in fm units. */
int vh_eos_table_synthetic(int n, double emin_gev, double emax_gev, double a, double hbarc,
                           double* e, double* p, double* cs2, double* t);
/* Ideal Gubser flow (q, tau0, central temperature in GeV): e, u^x, u^y at
 * tau0 and the velocity at tau0 - dtau (prevu) for the 2+1D grid. */
int vh_profile_gubser(int nx, int ny, double dx, double dy, double q, double tau0, double dtau,
                      double t0_gev, double a, double hbarc, double* e, double* ux, double* uy,
                      double* prevu4);
/* Isothermal freeze-out hypersurface of a boost-invariant run between two
 * consecutive time slices (no counterpart in the reference, which only stops
 * at the freeze-out temperature, NEWEST5/main.cpp:201-204).  t0, t1: the
 * temperature on the ghost-inclusive nx x ny grid at tau0 < tau1 (any unit,
 * the same as t_fo); u0, u1: u^tau, u^x, u^y there (3 fields).  The surface
 * T = t_fo of the samples' piecewise-linear interpolant is found by marching
 * tetrahedra over the space-time cubes between neighbouring interior cell
 * centres (six tetrahedra per cube); each triangle gives 9 doubles: its centroid (tau, x, y), the
 * covariant surface element dSigma_mu = tau eps_{mu nu lambda} dx^nu dx^lambda
 * / 2 per unit rapidity (mu = tau, x, y), pointing from the hot side to the
 * cold side, and u^tau, u^x, u^y interpolated there.  Writes at most cap
 * elements into out; *count receives the number found (VH_E_ARG when it
 * exceeds cap; cap = 0 with out = NULL only counts).  Host code. */
int vh_freezeout_2d(int nx, int ny, double dx, double dy, double tau0, double tau1, const double* t0,
                    const double* t1, const double* u0, const double* u1, double t_fo, double* out, long long cap,
                    long long* count);
/* Boltzmann Cooper-Frye spectrum E dN/d^3p at mid-rapidity from count
 * elements of vh_freezeout_2d (boost invariant, u^eta = 0; the rapidity
 * integral done with e^a K0(a), e^a K1(a) by the trapezoidal rule on their
 * integral representation, relative error within 4e-15, so that no factor
 * overflows at large p_T): out[a * nphi + b] at p_T = pt[a], azimuth
 * phi[b], for a hadron of mass and degeneracy at the surface temperature
 * t_fo (mass, momenta and t_fo in the same unit, e.g. fm^-1).  Host code. */
int vh_cooper_frye_2d(const double* elements, long long count, double t_fo, double mass, double degeneracy,
                      const double* pt, int npt, const double* phi, int nphi, double* out);
/* The same at rapidity y from count elements of vh_freezeout_3d (each at
 * its own eta; u^eta included).  Host code. */
int vh_cooper_frye_3d(const double* elements, long long count, double t_fo, double mass, double degeneracy, double y,
                      const double* pt, int npt, const double* phi, int nphi, double* out);
/* The same on a 3+1D Milne grid (nx x ny x nz cells of dx, dy, d eta):
 * marching 4-simplices (24 per space-time hypercube) give tetrahedra; each
 * gives 12 doubles: its centroid (tau, x, y, eta), dSigma_mu = tau
 * eps_{mu nu lambda rho} dx^nu dx^lambda dx^rho / 6 (mu = tau, x, y, eta),
 * hot to cold, and u^mu interpolated there (u0, u1: 4 fields). */
int vh_freezeout_3d(int nx, int ny, int nz, double dx, double dy, double dz, double tau0, double tau1,
                    const double* t0, const double* t1, const double* u0, const double* u1, double t_fo, double* out,
                    long long cap, long long* count);
/* The surfaces of vh_freezeout_2d and vh_freezeout_3d computed on the GPU
 * from device arrays (t0, t1: the ghost-inclusive slice, G doubles each;
 * u0, u1: 3 x G or 4 x G) into device memory out (cap elements of 9 or 12
 * doubles), element for element in the host functions' order: a count pass
 * over the space-time cubes, an exclusive scan, an emit pass.  cap = 0 with
 * out = NULL only counts.  Issued on stream (a cudaStream_t; NULL: the
 * legacy stream), which is synchronised to return *count; scratch comes from
 * the stream-ordered allocator.  Returns VH_E_ARG, with *count set, when
 * the surface has more than cap elements (the first cap are written). */
int vh_freezeout_2d_device(int nx, int ny, double dx, double dy, double tau0, double tau1, const double* t0,
                           const double* t1, const double* u0, const double* u1, double t_fo, double* out,
                           long long cap, long long* count, void* stream);
int vh_freezeout_3d_device(int nx, int ny, int nz, double dx, double dy, double dz, double tau0, double tau1,
                           const double* t0, const double* t1, const double* u0, const double* u1, double t_fo,
                           double* out, long long cap, long long* count, void* stream);
/* The surface T = t_fo swept by the handle's state since the last call,
 * on the GPU without host copies of the slices: T and u^mu of the current
 * state against those this call kept from the previous one (at its tau),
 * as vh_freezeout_2d_device (boost invariant) or vh_freezeout_3d_device
 * write it into device memory out (cap elements of 9 or 12 doubles).  The
 * first call after the state is set (vh_set_state, vh_init_profile,
 * vh_init_tmunu, vh_load_checkpoint) only keeps the slice and returns
 * *count = 0; a call between which no step ran returns VH_E_STATE.  When
 * the surface has more than cap elements the call returns VH_E_ARG with
 * *count set and keeps the previous slice, so that a call with a larger
 * out gets the same surface.  Milne grids only (VH_E_UNSUPPORTED on
 * Cartesian ones).  Call after each vh_step(h, 1) to follow the surface
 * through a run. */
int vh_freezeout_step(vh_handle* h, double t_fo, double* out, long long cap, long long* count);
/* vh_cooper_frye_2d and vh_cooper_frye_3d on the GPU: elements in device
 * memory (count x 9 or 12 doubles), momentum bins pt, phi and the result
 * out (npt x nphi) on the host; one block per bin sums the elements in a
 * fixed order.  Synchronises stream before returning. */
int vh_cooper_frye_2d_device(const double* elements, long long count, double t_fo, double mass, double degeneracy,
                             const double* pt, int npt, const double* phi, int nphi, double* out, void* stream);
int vh_cooper_frye_3d_device(const double* elements, long long count, double t_fo, double mass, double degeneracy,
                             double y, const double* pt, int npt, const double* phi, int nphi, double* out,
                             void* stream);
/* The viscous Gubser flow of the cold-plasma limit (the reference's
 * COLDPLASMA initial state, NEWEST5/init.h:489-512): conformal e = a T^4
 * with T = T^(rho)/tau, T^ = b sech(rho)^(2/3) cosh(k ln cosh rho)^(1/4),
 * k = 4/(3 sqrt 5), sinh rho = -(1 - q^2 tau^2 + q^2 r^2)/(2 q tau); Gubser
 * velocity; pi^{mu nu} from the de Sitter shear pi^eta_eta = -(4/3) a T^^4
 * tanh(k ln cosh rho)/sqrt 5, scaled by tau^-4 into Milne coordinates.
 * Writes e, u^x, u^y, pi5 (xx, yy, xy, x-eta, y-eta) at tau0 and prevu4 at
 * tau0 - dtau on the 2+1D ghost-inclusive grid.  The reference's values:
 * q = 1/fm, b = 1.21. */
int vh_profile_gubser_cold(int nx, int ny, double dx, double dy, double q, double tau0, double dtau, double b,
                           double a, double* e, double* ux, double* uy, double* pi5, double* prevu4);
/* Israel-Stewart Gubser flow (the reference's viscous Gubser test, whose
 * initial table init/tempbin-23F.dat it reads at NEWEST5/init.h:419-459 and
 * does not ship): conformal e = a T^4, eta/s constant, tau_pi = 5 eta/(e+P)
 * (NEWEST5/maindef.h:338-339).  T^ = tau T and P = tau^2 pi^{eta eta}/(e+P)
 * solve, in the de Sitter time rho (sinh rho = -(1 - q^2 tau^2 +
 * q^2 r^2)/(2 q tau)),
 *   d ln T^/d rho = -(2/3) tanh rho + (1/3) P tanh rho,
 *   dP/d rho = -(4/3) P^2 tanh rho - P T^/(5 eta/s) + (4/15) tanh rho,
 * fixed by T = t0_gev and P = p0 at the grid centre at tau0 (RK4, step 1e-3
 * in rho).  Writes e, u^x, u^y (Gubser velocity) and pi5 (xx, yy, xy,
 * x-eta, y-eta: w P along eta, -w P/2 along the two transverse rest-frame
 * directions) at tau0 and prevu4 at tau0 - dtau on the 2+1D ghost-inclusive
 * grid.  The reference's shipped table (init/tempbin-8.7z: q = 1/fm,
 * T = 1.2 fm^-1 and P = 0 at tau0 = 1 fm/c, eta/s = 0.2) is this solution. */
int vh_profile_gubser_is(int nx, int ny, double dx, double dy, double q, double tau0, double dtau, double t0_gev,
                         double p0, double etas, double a, double hbarc, double* e, double* ux, double* uy,
                         double* pi5, double* prevu4);
/* Monte-Carlo Glauber energy density (two Woods-Saxon nuclei): A nucleons
 * per nucleus, radius R, diffuseness aws, hard core dmin, impact parameter
 * b, sigma_nn (fm^2), Gaussian width w per participant, peak e in GeV/fm^3,
 * eta plateau half-width and Gaussian tail width, a floor efloor_gev
 * (GeV/fm^3) under which no cell starts; seed.  Writes e (fm^-4) on the
 * ghost-inclusive grid and returns the participant count in *npart. */
int vh_profile_glauber(int nx, int ny, int nz, int boost_invariant, double dx, double dy, double dz,
                       int A, double R, double aws, double dmin, double b, double sigma_nn,
                       double w, double epeak_gev, double eta_flat, double eta_sigma, double efloor_gev,
                       double hbarc, uint64_t seed, double* e, int* npart);

#ifdef __cplusplus
}
#endif
#endif
