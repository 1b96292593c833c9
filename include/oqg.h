/*
 * oqg.h -- C ABI of the B200 implementation of OpenQG's per-timestep
 * quasi-geostrophic core (module `core`, subroutine `step_qg`).
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns an int status (OQG_OK == 0).  No call aborts the process; the
 * reference's `stop 1` paths (util/linalg.F90:124-136, qg/modes.F90:148-161)
 * become nonzero status codes, and oqg_last_error() gives the message.
 *
 * Arrays crossing this boundary are FP64 in the reference's Fortran
 * column-major layout: element (i, j, k) of an (nxp, nyp, nl) array is at
 * offset i + nxp*(j + nyp*k), with 0-based i, j, k.  Host buffers are owned
 * by the caller.  A handle owns one CUDA stream; a handle is not thread-safe,
 * distinct handles are.
 *
 * Reference interface replaced (file:line within BreakawayLabs/openqg):
 *   step_qg(tdt, ent, wekp, txis, txin, qg)        src/qg/core.F90:16-33
 *   init_qg(go, bcco, delek, ah2, ah4, gp, rho,...) src/qg/qg.F90:60-103
 *   init_pv / qcomp                                 src/qg/vorsubs.F90:17-56
 *   init_constraint / init_mass_constr              src/qg/constraint.F90:80-165
 *   suppress_comp_mode                              src/driver.F90:174-189
 *   restart_qg / save_qg state (p, pm)              src/state.F90:29-112
 *   solve_inhomog_eqn / generate_homog_soln         src/qg/inhomog.F90:146-168
 *   ekman_from_tau                                  src/coupler/ekman.F90:53-83
 *   qg_diagno (ekei, sfmin, sfmax, circ)            src/diagnostics/qg_monitor.F90:289-376
 *   qg_diagno (the full monitor record)             src/diagnostics/qg_monitor.F90:219-383
 *   valids (p, q and Ekman-pumping bounds)          src/diagnostics/valsubs.F90:46-139
 */
#ifndef OQG_H
#define OQG_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OQG_MAX_NL 8

/* status codes */
#define OQG_OK           0
#define OQG_EINVAL       1  /* bad argument or parameter set            */
#define OQG_ECUDA        2  /* CUDA runtime error                        */
#define OQG_ENAN         3  /* non-finite value found in the state       */
#define OQG_ETIMEOUT     4  /* a bounded device wait ran out             */
#define OQG_EUNSUPPORTED 5  /* size or mode this build does not handle   */
#define OQG_ESETUP       6  /* init-time check failed (e.g. mode matrix
                               product not the identity, singular LU)   */
#define OQG_ENODEV       7  /* no CUDA device                            */
#define OQG_ESCRATCH     8  /* problem larger than a fixed scratch area  */

/* precision modes */
#define OQG_FP64   0  /* everything FP64, the reference's arithmetic            */
#define OQG_MIXED  1  /* FP32 state, stencils, Jacobian and x-transforms; FP64
                         vertical-mode projection, tridiagonal solves and
                         constraint / area integrals                          */

/*
 * Parameters of one QG basin: the fields init_qg receives (qg.F90:60-70)
 * plus the box geometry (glam/box.F90:11-41) and topography (topog.F90:20-21).
 * Lengths in m, times in s, like the reference.
 */
typedef struct oqg_params {
    int    nxp, nyp, nl;      /* p-grid points and layers (nxp = nxt+1)        */
    int    cyclic;            /* 1: zonally periodic channel; 0: closed box    */
    double dx, dy;            /* grid spacing                                   */
    double fnot, beta;        /* f0 and beta of the beta-plane                  */
    int    dz_sign;           /* -1 ocean, +1 atmosphere (basin.F90:36,129)     */
    int    tau_sign;          /* +1 ocean, -1 atmosphere (basin.F90:62,158)     */
    double h[OQG_MAX_NL];     /* layer thicknesses, nl used                     */
    double gp[OQG_MAX_NL];    /* reduced gravities, nl-1 used                   */
    double ah2[OQG_MAX_NL];   /* Laplacian viscosity per layer                  */
    double ah4[OQG_MAX_NL];   /* biharmonic viscosity per layer                 */
    double bcco;              /* mixed boundary coefficient (0 free slip,
                                 large -> no slip)                              */
    double delek;             /* bottom Ekman layer thickness                   */
    double rho;               /* density used by the diagnostics                */
    int    k_topo;            /* 1-based layer carrying topography and drag     */
    int    precision;         /* OQG_FP64 or OQG_MIXED                          */
    int    suppress_period;   /* average time levels when mod(nt-1,period)==0
                                 (openqg.F90:485-487); 0 never                  */
    const double *ddyn;       /* (nxp, nyp) dynamic topography; NULL = flat     */
} oqg_params;

typedef struct oqg_handle oqg_handle;

/* Message of the last failure on this thread ("" if none). */
const char *oqg_last_error(void);

/* Library and device description (for logs): writes a NUL-terminated string. */
int oqg_version(char *buf, int buflen);

/* init_qg (qg.F90:60-103): vertical modes, Helmholtz tables and homogeneous
 * solutions are computed, uploaded and kept on the current CUDA device.
 * State starts at zero, forcing at zero, step counter nt = 0. */
int oqg_create(const oqg_params *prm, oqg_handle **out);
int oqg_destroy(oqg_handle *h);

/* Restart semantics (openqg.F90:233-243, state.F90:29-44): takes p, pm
 * (nxp,nyp,nl) and recomputes q, qm (init_pv), the channel momentum
 * constraints (init_constraint) and the mass constraint (init_mass_constr). */
int oqg_set_state(oqg_handle *h, const double *p, const double *pm);

/* Full state: p, pm, q, qm (nxp,nyp,nl) and the constraint scalars
 * dpi, dpip (nl-1) and cs, cn, csp, cnp (nl; ignored for a box). */
int oqg_set_state_full(oqg_handle *h, const double *p, const double *pm,
                       const double *q, const double *qm,
                       const double *dpi, const double *dpip,
                       const double *cs, const double *cn,
                       const double *csp, const double *cnp);

/* Copies the state out; any pointer may be NULL to skip that field. */
int oqg_get_state(oqg_handle *h, double *p, double *pm, double *q, double *qm);
int oqg_get_constraints(oqg_handle *h, double *dpi, double *dpip,
                        double *cs, double *cn, double *csp, double *cnp);

/* Copies layer k (0-based) of p out: the p(:,:,1) exchange of
 * driver.F90:99-101. */
int oqg_get_p_layer(oqg_handle *h, int k, double *out);

/* Forcing of step_qg: wekp (nxp,nyp), ent (nxp,nyp,nl-1) or NULL for zero
 * entrainment, and the channel wind-stress integrals txis, txin.  Stored on
 * the device and reused by every step until set again.  A closed box's step
 * reads ent(:,:,1) alone (vorticity.F90:71-72, pressure.F90:52-53), so for a
 * box only that layer is copied (the device keeps zeros in the others); a
 * channel copies every layer (its momentum constraints read layer 2's wall
 * rows, vorticity.F90:88-93). */
int oqg_set_forcing(oqg_handle *h, const double *wekp, const double *ent,
                    double txis, double txin);

/* Runs nsteps calls of step_qg(tdt, ...) (core.F90:16-33).  Before step nt
 * (1-based, counted by the handle) returns, suppress_comp_mode is applied when
 * suppress_period > 0 and mod(nt-1, suppress_period) == 0, as the run loop
 * does (openqg.F90:485-487, driver.F90:78-85).  Steps are queued on the
 * handle's stream; the call returns after they are queued (see oqg_sync). */
int oqg_step(oqg_handle *h, double tdt, int nsteps);

/* Sets the step counter (number of steps already taken, nt-1 of the next). */
int oqg_set_step_index(oqg_handle *h, long long steps_done);
int oqg_get_step_index(oqg_handle *h, long long *steps_done);

/* suppress_comp_mode (driver.F90:174-189) applied once, now. */
int oqg_suppress(oqg_handle *h);

/* Waits for the handle's stream; reports a deferred device error and clears
 * it: OQG_ETIMEOUT when a bounded device wait ran out (that step's results
 * are invalid; set the state again before stepping on), OQG_ECUDA for any
 * other device error.  No counterpart in the reference (its step cannot
 * fail: errors abort with stop 1, util/linalg.F90:130-134). */
int oqg_sync(oqg_handle *h);

/* Test hook of the failure detection (no counterpart in the reference): the
 * number of polls a kernel's first wait for a tile load makes before it
 * reports a timeout.  polls = 0 makes every such wait run out at once (the
 * kernel then drains its copies in flight with the full limit, sets the
 * error word and returns); polls < 0 restores the default, 2^22. */
int oqg_set_wait_limit(oqg_handle *h, long long polls);

/* Device validity scan of p and q (the role of valids, valsubs.F90:46-139):
 * *bad = number of non-finite values found. */
int oqg_check_finite(oqg_handle *h, long long *bad);

/* Diagnostics of qg_diagno (qg_monitor.F90:289-376), each of length nl:
 * layer kinetic energy ekei, stream-function extrema sfmin/sfmax (Sv) and the
 * total circulation circ (Sv).  Any pointer may be NULL. */
int oqg_diag(oqg_handle *h, double *ekei, double *sfmin, double *sfmax,
             double *circ);

/* oqg_diag without any allocation: no counterpart in the reference.
 *
 * For callers that must not allocate device memory at call time: a host
 * whose GPU memory is wholly reserved by another allocator (a framework's
 * caching pool, a fixed partition of the device), or a monitor that runs
 * between steps of a time-critical loop, where cudaMalloc/cudaFree would
 * block on or synchronise the device.  Results equal oqg_diag's (the kinetic
 * energy to rounding: rows are summed first, then layers).
 *
 * Its scratch is a 256 KiB array compiled into the library (32768 doubles);
 * a basin fits when 40 + 4*nl*nyp <= 32768 (nl*nyp <= 8182), otherwise the
 * call returns OQG_ESCRATCH and does nothing.  It calls no cudaMalloc,
 * cudaFree or other allocating routine, and reports failures by status code
 * alone (oqg_last_error is not updated).
 *
 * The first call on a device looks up the array's address on that device
 * (the handle's device must be current; OQG_EINVAL otherwise), which may make
 * the CUDA runtime load the library's device code: make that first call
 * before any stream capture.  Every call clears the scratch's completion
 * counter on the handle's stream before its kernel.  There is one array per
 * device: calls that overlap in time on the same device (any handles,
 * streams or host threads) race on it and corrupt each other's results, so
 * callers must serialise them. */
int oqg_diag_noalloc(oqg_handle *h, double *ekei, double *sfmin, double *sfmax,
                     double *circ);

/* The monitor record of qg_diagno (qg_monitor.F90:219-383): forcing means,
 * interface displacement, energetics, jet, transports and stream-function
 * extrema; arrays of length nl (nl-1 for the interface quantities).  tsec and
 * et2m carry state from one call to the next (pket is the rate of change of
 * the interface potential energy since the previous call), as in the
 * reference's qg_monitor_type. */
typedef struct oqg_qg_monitor {
    double tsec;                       /* time of the previous call (s)         */
    double wepm, wapm;                 /* mean Ekman pumping, mean |pumping|    */
    double entm, enam;                 /* mean entrainment, mean |entrainment|  */
    double etam[OQG_MAX_NL], et2m[OQG_MAX_NL], pket[OQG_MAX_NL];
    double pken;                       /* rho gp1 <eta1 ent1>                   */
    double utau;                       /* wind work rho int(tau . u_geo)        */
    double pavg[OQG_MAX_NL], qavg[OQG_MAX_NL];
    double ah2d[OQG_MAX_NL], ah4d[OQG_MAX_NL];   /* viscous dissipation        */
    double ekei[OQG_MAX_NL];                     /* layer kinetic energy       */
    double val[OQG_MAX_NL];                      /* jet strength               */
    int    pos[OQG_MAX_NL];                      /* jet row (1-based)          */
    double circ[OQG_MAX_NL], ctot;               /* circulation (Sv)           */
    double btdg;                                 /* bottom Ekman drag          */
    double sfmin[OQG_MAX_NL], sfmax[OQG_MAX_NL]; /* stream-function extrema    */
    double ermas[OQG_MAX_NL], emfr[OQG_MAX_NL];  /* channel continuity check   */
} oqg_qg_monitor;

/* qg_diagno (qg_monitor.F90:219-383) on the device from the current state
 * and forcing: taux, tauy (nxp, nyp) are the wind stress the Ekman pumping
 * came from (NULL: utau = 0); tsec the model time; tdt the leapfrog step (for
 * the channel continuity check).  mon is read (tsec, et2m) and written. */
int oqg_diagno(oqg_handle *h, const double *taux, const double *tauy, double tsec,
               double tdt, oqg_qg_monitor *mon);

/* The QG part of the validity scan valids (valsubs.F90:46-139): extremes of
 * p and q over all layers and of the Ekman pumping wekp, each compared with
 * its bound (|min| or |max| >= bound is invalid, as in the reference).
 * ext[6] = pmin, pmax, qmin, qmax, wmin, wmax; *ok = 1 when all are valid.
 * Non-finite values also make *ok = 0 (the reference's comparisons let a
 * NaN pass); *nonfinite counts them.  Pointers other than ok may be NULL. */
int oqg_valids(oqg_handle *h, double pext, double qext, double wext, double *ext,
               long long *nonfinite, int *ok);

/* int_P_dA (numerics.F90:165-204): the trapezoid-rule area integral of a
 * field (nxp, nyp) on the basin's grid, computed on the device with the
 * compensated summation the step's mass-constraint and area integrals use. */
int oqg_int_P_dA(oqg_handle *h, const double *field, double *out);

/* solve_inhomog_eqn (inhomog.F90:156-168): (Del^2 - rdm2(m)) out = rhs with
 * out = 0 on solid boundaries; m is the 1-based mode; rhs, out (nxp, nyp). */
int oqg_solve_inhomog(oqg_handle *h, int m, const double *rhs, double *out);

/* generate_homog_soln (inhomog.F90:146-154): out = L + rdm2(m)*solve(L). */
int oqg_generate_homog_soln(oqg_handle *h, int m, const double *L, double *out);

/* Vertical-mode tables of eigmod (modes.F90:46-219); amat, ctl2m, ctm2l are
 * (nl, nl) column-major, rdm2 has nl entries.  Any pointer may be NULL. */
int oqg_get_modes(oqg_handle *h, double *amat, double *rdm2,
                  double *ctl2m, double *ctm2l);

/* ekman_from_tau (ekman.F90:53-83) for a basin with these parameters:
 * taux, tauy (nxp, nyp) kinematic stress -> wekp (nxp, nyp) Ekman velocity at
 * p points and, for a channel, the boundary integrals txis, txin. */
int oqg_ekman_from_tau(const oqg_params *prm, const double *taux,
                       const double *tauy, double *wekp,
                       double *txis, double *txin);

/* Device pointers of the state, for zero-copy use by the PyTorch extension:
 * p, pm, q, qm as (nl, nyp, pitch) arrays of the handle's storage type
 * (FP64 or, in OQG_MIXED, FP32); *pitch is the row pitch in elements.  In
 * OQG_MIXED q and qm hold q - beta*yprel(j) (the planetary vorticity is kept
 * out of the FP32 values; oqg_get_state adds it back). */
int oqg_device_state(oqg_handle *h, void **p, void **pm, void **q, void **qm,
                     int *pitch, int *elem_bytes);

/* Runs nsteps steps as separate launches with CUDA events between the
 * kernels of each step, on the handle's stream, and returns the mean device
 * time per launch (ms) of each: ms[0] vorticity step + modal RHS, ms[1]
 * forward x-transform, ms[2] y-solve, ms[3] inverse x-transform (with the
 * scalar phase, and with the assembly when one kernel does both), ms[4] the
 * assembly when it runs as a launch of its own (oqg_set_xinv_sep), else 0.
 * ms holds 5 values.  For measurement; the state advances normally. */
int oqg_profile_phases(oqg_handle *h, double tdt, int nsteps, double *ms);

/* CUDA stream of the handle (a cudaStream_t). */
int oqg_stream(oqg_handle *h, void **stream);

/* Kernel launches of one model step: 5 for a closed box (vorticity, forward
 * transform, y-solve, inverse transform, assembly), 4 with the inverse
 * transform and the assembly in one kernel (a channel's default, or after
 * oqg_set_xinv_sep(h, 0)). */
int oqg_step_launches(oqg_handle *h, int *launches);

/* The launch floor of the step chain: nsteps steps of launches with the
 * step kernels' grids, blocks, shared-memory sizes and dependent-launch
 * chaining but no work, replayed from a CUDA graph on the handle's stream;
 * the device time per step in microseconds.  For measurement: it tells how
 * much of a step a single persistent launch could save at most. */
int oqg_launch_floor(oqg_handle *h, int nsteps, double *us_per_step);

/* Measures the vorticity kernel's tile heights (8, 12 and 16 rows of 60 columns)
 * on the device: for each, nsteps (>= 2) steps of tdt from the handle's
 * current state, timed with CUDA events; keeps the fastest, restores the
 * state, and records the height for the basin's shape and precision, so
 * handles created afterwards in this process start from it.  *best_vty
 * (may be NULL) gets the height; ms (NULL or >= 18 doubles) gets the time
 * per step of each height at index height.  Results do not depend on the
 * height (each point is computed the same way in any tile). */
int oqg_autotune(oqg_handle *h, double tdt, int nsteps, int *best_vty, double *ms);
/* Current tile height of the vorticity kernel. */
int oqg_get_vty(oqg_handle *h, int *vty);

/* The y-solve's warps per column (1, 2 or 4): oqg_create picks enough for
 * about 20 warps per SM while each lane keeps 4 to 8 rows; this measures the
 * three on the device like oqg_autotune (nsteps steps of tdt from the
 * current state, restored) and keeps the fastest.  ms[0..2]: ms per step
 * with 1, 2 and 4 warps.  Results agree to rounding (the scan's
 * association changes with the split). */
int oqg_autotune_ysolve(oqg_handle *h, double tdt, int nsteps, int *best_warps, double *ms);
/* Current warps per y-solve column. */
int oqg_get_ysolve_warps(oqg_handle *h, int *warps);
/* Fix the vorticity tile height (8, 12 or 16) or the y-solve's warps per
 * column (1, 2 or 4) without measuring, e.g. from an earlier oqg_autotune
 * on the same GPU; OQG_EINVAL for other values. */
int oqg_set_vty(oqg_handle *h, int vty);
int oqg_set_ysolve_warps(oqg_handle *h, int warps);
/* The inverse transforms as a launch shaped like the forward
 * one (k_xinv_rows, which also runs the step's scalar phase once) and a
 * one-pass assembly (k_xinv_asm), instead of one kernel that transforms and
 * assembles in shared memory.  On by default for boxes, off for channels;
 * it cannot be turned off where the modal rows do not fit in shared memory
 * (1025 points wide and more: OQG_EUNSUPPORTED). */
int oqg_set_xinv_sep(oqg_handle *h, int on);
int oqg_get_xinv_sep(oqg_handle *h, int *on);
/* Measures the two forms of the inverse transform and assembly (one kernel,
 * or two launches) like oqg_autotune and keeps the faster; ms[0]: one
 * kernel, ms[1]: two launches (ms per step; -1 where a form is not
 * available: wide grids keep the two launches and return at once). */
int oqg_autotune_xinv(oqg_handle *h, double tdt, int nsteps, int *best_sep, double *ms);

/* ---------------------------------------------------------------------
 * Ensembles: many independent basins of uneven size stepped together by one
 * launch per phase (captured in a CUDA graph).  Members keep the semantics of
 * a single handle and match its results to rounding; they must share nl and
 * precision, and be all closed boxes or all channels (OQG_EINVAL /
 * OQG_EUNSUPPORTED otherwise).  Per-member calls (set_state, set_forcing,
 * get_state) wait for the ensemble's stream first.  member is 0-based.
 * ------------------------------------------------------------------- */
typedef struct oqg_ensemble oqg_ensemble;

int oqg_ensemble_create(const oqg_params *members, int nmembers,
                        oqg_ensemble **out);
int oqg_ensemble_destroy(oqg_ensemble *e);
int oqg_ensemble_set_state(oqg_ensemble *e, int member,
                           const double *p, const double *pm);
int oqg_ensemble_get_state(oqg_ensemble *e, int member, double *p,
                           double *pm, double *q, double *qm);
int oqg_ensemble_set_forcing(oqg_ensemble *e, int member, const double *wekp,
                             const double *ent, double txis, double txin);
/* tdt[member] per member; nsteps for all. */
int oqg_ensemble_step(oqg_ensemble *e, const double *tdt, int nsteps);
int oqg_ensemble_sync(oqg_ensemble *e);
/* The CUDA stream (cudaStream_t) the ensemble's steps run on. */
int oqg_ensemble_stream(oqg_ensemble *e, void **stream);
/* oqg_autotune for an ensemble: one vorticity tile height for all members,
 * measured over nsteps steps (tdt per member) from the members' current
 * states, which are restored.  best_vty / ms as for oqg_autotune. */
int oqg_ensemble_autotune(oqg_ensemble *e, const double *tdt, int nsteps, int *best_vty, double *ms);

/* ---------------------------------------------------------------------
 * The ocean half of the coupler on the device: the Ekman fields from the
 * wind stress and the ocean mixed-layer step, writing the QG handle's
 * forcing (wekp, ent) in place, so the layer-1 pressure, the pumping and the
 * entrainment never cross to the host.  Replaces, for a closed box:
 *   ekman_from_tau                          src/coupler/ekman.F90:53-83
 *   step_oml (with adv_diff, del2_T, ...)   src/mixed/omlsubs.F90:69-119,
 *                                           src/mixed/mixed_layer.F90:16-95
 *   the ocean step's exchange               src/driver.F90:95-107
 * ------------------------------------------------------------------- */
typedef struct oqg_oml oqg_oml;

/* init_ocean_ml (omlsubs.F90:27-67) and the temp_type fields it reads. */
typedef struct oqg_oml_params {
    double hm;          /* mixed-layer depth (m), the box's hm               */
    double rho_cp;      /* rho * cp of sea water (J m^-3 K^-1)              */
    double t1_rel;      /* T_bar - T(1) (K)                                  */
    double dt_12;       /* T(1) - T(2) (K)                                   */
    double st2d, st4d;  /* Laplacian / biharmonic sst diffusivities          */
    double ycexp;       /* coefficient of the geostrophic advection          */
    int    fluxn, fluxs;/* heat-flux condition at the northern / southern wall */
    double nval, sval;  /* the wall temperatures of those conditions (K)     */
} oqg_oml_params;

/* The mixed layer of the basin of handle qg (a closed box); sst starts at
 * zero (init_mixed, mixed.F90:73-99).  OQG_EINVAL for a heat-flux condition
 * on the wrong hemisphere's wall, as the reference's init stops. */
int oqg_oml_create(oqg_handle *qg, const oqg_oml_params *prm, oqg_oml **out);
/* Frees the mixed layer; it does not touch the handle, so it may come before
 * or after oqg_destroy of qg.  No other call may follow oqg_destroy of qg. */
int oqg_oml_destroy(oqg_oml *m);
/* sst and its lagged value, (nxt, nyt) = (nxp-1, nyp-1), host or device. */
int oqg_oml_set_sst(oqg_oml *m, const double *sst, const double *sstm);
int oqg_oml_get_sst(oqg_oml *m, double *sst, double *sstm);
/* One ocean coupling step before step_qg (driver.F90:95-103): ekman_from_tau
 * of taux, tauy (nxp, nyp) with the box's hm, then step_oml with the handle's
 * current p(:,:,1) and the net heat flux fnetoc (nxt, nyt).  The handle's
 * wekp becomes map_T_to_P(wekt); when compute_ent, its ent becomes the
 * layer 1/2 entrainment (other layers zero), otherwise ent is kept.
 * Arrays in host or device memory.  taux = tauy = NULL: the stress that
 * oqg_xforc last computed on the device; fnetoc = NULL: the flux that
 * oqg_compute_forcing last computed on the device (zero before the first).
 * The call returns once its copies are done; with nothing to copy it returns
 * without waiting for the device (the work stays queued on the stream). */
int oqg_ocean_forcing(oqg_oml *m, const double *taux, const double *tauy,
                      const double *fnetoc, int compute_ent, double tdto);
/* The handle's forcing, wekp (nxp, nyp) and ent (nxp, nyp, nl-1), copied
 * to host arrays (either may be NULL); for a box the layers after the first
 * are the zeros the step reads in their place. */
int oqg_get_forcing(oqg_handle *h, double *wekp, double *ent);

/* The atmosphere half: the Ekman fields of a channel and the atmospheric
 * mixed-layer step, writing the atmosphere handle's wekp, ent, txis, txin.
 * Replaces, for a zonally periodic channel:
 *   ekman_from_tau (with txis, txin)        src/coupler/ekman.F90:53-83
 *   step_aml, compute_new_aml,
 *   compute_atmos_entrainment               src/mixed/amlsubs.F90:184-326
 *   the atmosphere step's exchange          src/driver.F90:113-143
 * The radiation scheme's start-up (radiat, radsubs.F90:116-157) and the
 * entrainment coefficients (init_entrain_coeff, set_xc1ast) stay with the
 * caller: their results are passed in.  The per-step fluxes (compute_forcing)
 * and both basins' stress (xforc) run on the device, below. */
typedef struct oqg_aml oqg_aml;

/* init_atmos_ml (amlsubs.F90:61-98) and the coefficients it derives. */
typedef struct oqg_aml_params {
    double hm;              /* the box's mixed-layer depth (m)               */
    double rho_cp;          /* rho * cp of air                               */
    double t1_rel, dt_12;   /* T_bar - T(1), T(1) - T(2) (K)                 */
    double hmamin, hmadmp;  /* height floor (m) and damping                  */
    double xcexp;           /* entrainment coupling coefficient              */
    double at2d, at4d;      /* temperature diffusivities                     */
    double ahmd;            /* height diffusivity                            */
    double bface, dface;    /* entrainment coefficients (init_entrain_coeff) */
    double cdat;            /* drag coefficient of the stress (windstress.F90) */
    double aface[OQG_MAX_NL];   /* of eta(1..nl-1)                           */
} oqg_aml_params;

/* The atmospheric mixed layer of channel handle qg; xc1ast (nxt, nyt) from
 * set_xc1ast and the topography dtop (nxp, nyp) or NULL (flat), host or
 * device memory.  ast starts at 0 and hmixa at hm (init_atmos_ml). */
int oqg_aml_create(oqg_handle *qg, const oqg_aml_params *prm, const double *xc1ast,
                   const double *dtop, oqg_aml **out);
/* Frees the mixed layer without touching the handle (either order). */
int oqg_aml_destroy(oqg_aml *m);
/* ast, its lagged value, hmixa and its lagged value, (nxt, nyt) each. */
int oqg_aml_set_state(oqg_aml *m, const double *ast, const double *astm,
                      const double *hmixa, const double *hmixam);
int oqg_aml_get_state(oqg_aml *m, double *ast, double *astm, double *hmixa,
                      double *hmixam);
/* One atmosphere coupling step before step_qg (driver.F90:113-143):
 * ekman_from_tau of taux, tauy (nxp, nyp) with the box's hm, then step_aml
 * with the handle's current p(:,:,1), eta from its lagged pressure
 * (pm_k - pm_{k+1}) / gp_k, and the net heat flux fnetat (nxt, nyt).  The
 * handle's wekp, txis, txin become the Ekman forcing; when compute_ent, its
 * ent becomes the layer 1/2 entrainment (other layers zero).  taux = tauy =
 * NULL: the stress that oqg_xforc last computed on the device; fnetat = NULL:
 * the flux that oqg_compute_forcing last computed (zero before the first). */
int oqg_atmos_forcing(oqg_aml *m, const double *taux, const double *tauy,
                      const double *fnetat, int compute_ent, double tdta);

/* Couples an ocean mixed layer to an atmospheric one (NULL unlinks), for
 * oqg_xforc and oqg_compute_forcing below: raoro = rho_atmosphere /
 * rho_ocean.  The ocean grid must hold whole atmospheric cells (load_grid,
 * grid.F90:36-59); the ocean sits at the channel's western end (nx1 = 1),
 * centred in y.  The atmosphere must outlive the link. */
int oqg_oml_couple(oqg_oml *m, oqg_aml *a, double raoro);

/* Both basins' wind stress from the atmosphere's lagged layer-1 pressure, on
 * the device, held for the forcing calls that follow with NULL stresses
 * (xforc, windstress.F90:102-148, the case without the ocean-velocity
 * dependence; the reference calls it at each ocean step, driver.F90:47-54):
 * the atmosphere's by the quadratic drag law at its p points; the ocean's,
 * when o is given (coupled to a), from the atmospheric geostrophic velocity
 * and its derivatives over the ocean interpolated bicubically to the ocean's
 * p points (compute_windstress, atmos_geos_vel, atmos_windstress;
 * windstress.F90:150-314, bicubic.F90) with the atmosphere's cdat and hm,
 * times raoro.  The two handles' streams are ordered around the read of the
 * pressure (CUDA events). */
int oqg_xforc(oqg_aml *a, oqg_oml *o);
/* tau_udiff (windstress.F90:24-34, 255-276) on or off for the coupled pair
 * (off at creation): the stress then follows the difference of the
 * atmospheric and the ocean's lagged geostrophic surface velocity, the drag
 * factor includes both mixed layers (cdat / f0a (1 / hma + raoro / hmo)),
 * and the atmosphere's stress at the p points the two grids share is the
 * ocean-resolution one (before raoro), as compute_windstress writes it. */
int oqg_oml_tau_udiff(oqg_oml *o, int on);

/* The radiation coefficients compute_forcing reads (radiate_type,
 * radsubs.F90:15-54), the derived values radiat computes at start-up. */
typedef struct oqg_rad_coeffs {
    double fspco;      /* signed perturbation forcing amplitude (W m^-2)     */
    double xlamda;     /* sensible + latent transfer coefficient (W m^-2 K^-1) */
    double d0up;       /* D0up: ocean mixed-layer upward radiation per K     */
    double dmdown;     /* Dmdown: atmospheric mixed-layer downward, per K    */
    double dup0;       /* Dup(0): atmospheric mixed-layer upward, per K      */
    double aup00;      /* Aup(0,0)                                           */
    double adown10;    /* Adown(1,0)                                         */
    double adown11;    /* Adown(1,1)                                         */
} oqg_rad_coeffs;

/* ---------------------------------------------------------------------
 * The radiation scheme's start-up on the host: the mean radiative balance
 * of the coupled atmosphere and the linearised coefficients that
 * compute_forcing and the mixed layers read.  Replaces:
 *   load_rad, radiat and its helpers      src/mixed/radsubs.F90:63-674
 *   init_temp_from_rad, zonal_temp        src/mixed/mixed.F90:102-151
 *   sin_lat                               src/glam/numerics.F90:516-525
 *   init_entrain_coeff, set_xc1ast        src/mixed/amlsubs.F90:100-182
 * Host code only; no device is touched.
 * ------------------------------------------------------------------- */

/* load_rad's inputs (radsubs.F90:63-94). */
typedef struct oqg_rad_params {
    double fsbar;                 /* background forcing amplitude (< 0, W m^-2)    */
    double fspamp;                /* perturbation forcing amplitude (>= 0, W m^-2) */
    double gamma;                 /* adiabatic lapse rate (K m^-1)                  */
    double xlamda;                /* sensible + latent transfer (W m^-2 K^-1)       */
    double zopt[OQG_MAX_NL + 1];  /* optical depths: mixed layer, layers 1..nl (m)  */
    double tabsat[OQG_MAX_NL];    /* the layers' absolute temperatures T_abs (K)    */
} oqg_rad_params;

/* radiat's results (radsubs.F90:116-157). */
typedef struct oqg_rad_state {
    oqg_rad_coeffs c;                        /* the values compute_forcing reads      */
    double aup[OQG_MAX_NL + 1][OQG_MAX_NL];  /* Aup(k, l), k = 0..nl, l = 0..nl-1     */
    double adown[OQG_MAX_NL][OQG_MAX_NL];    /* Adown(k, l) at [k-1][l], k = 1..nl    */
    double dup[OQG_MAX_NL + 1];              /* Dup(0..nl)                            */
    double rbetat[OQG_MAX_NL];               /* rbetat(1..nl-1) at [k-1]              */
    double rbtmat, rbtmoc;                   /* balance coefficients of Tm' (atm, ocn) */
    double atm_tmbar, ocn_tmbar;             /* mean mixed-layer temperatures (K)     */
} oqg_rad_state;

/* load_rad + radiat for an atmosphere of nl layers of thicknesses h, mixed
 * layer depth hm, Coriolis parameter fnot (the sign of fspco): the layers'
 * transmissivities, the mean up- and downgoing radiation (trapezoidal rule
 * on 10001 points), the mixed layers' mean temperatures (fixed-point
 * iterations to 1e-13 K), the mean fluxes, the perturbation coefficients and
 * the radiative-balance coefficients (an nl x nl LU solve).  OQG_EINVAL for
 * fspamp < 0, as load_rad stops; OQG_ESETUP when an iteration does not
 * converge in 200 steps or the balance matrix is singular. */
int oqg_radiat(int nl, const double *h, double hm, double fnot, const oqg_rad_params *p, oqg_rad_state *out);

/* init_entrain_coeff (amlsubs.F90:100-131): the entrainment coefficients of
 * interface 1, aface(1..nl-1) into aface[0..nl-2], bface, dface, from the
 * radiation coefficients, rho_cp of air and dt_12 = T(1) - T(2). */
int oqg_entrain_coeff(int nl, double rho_cp, double dt_12, const oqg_rad_state *rad, double *aface, double *bface,
                      double *dface);

/* zonal_temp (mixed.F90:144-151, sin_lat) at the nyt T rows of a basin whose
 * first p row is at y0 with spacing dy: -sign(dT_NS, fnot) / 2 *
 * sin(pi / 2 (y - yc) / (yn - yc)), yc the middle and yn the northern edge of
 * the atmosphere's y range [ya0, ya0 + yla] (init_temp_from_rad), dT_NS =
 * |rbtm * fspco|.  set_xc1ast's field is this profile on the atmosphere's
 * rows, repeated along x; the ocean's wall temperatures are its first and
 * last values on the ocean's rows (omlsubs.F90:38-41). */
int oqg_zonal_temp(int nyt, double y0, double dy, double fnot, double ya0, double yla, double dt_ns, double *out);

/* The net diabatic forcing of both mixed layers on the device, from the
 * lagged sst, the atmosphere's lagged temperature and height, eta_1 of its
 * lagged pressure and its topography (compute_forcing, forcing.F90:18-99;
 * the reference calls it at each ocean step before step_aml, driver.F90:
 * 133-137): the atmospheric temperature interpolated bilinearly to the
 * ocean's T points (bilint, numerics.F90:528-589), the ocean's flux and the
 * atmosphere's with the ocean cells' upward fluxes summed into the
 * atmospheric cells above them.  Held for the forcing calls that follow
 * with NULL fluxes.  o must be coupled (oqg_oml_couple). */
int oqg_compute_forcing(oqg_oml *o, const oqg_rad_coeffs *rad);
/* The fluxes held on the device, fnetoc (nxt, nyt) of the ocean and fnetat
 * (nxt, nyt) of the coupled atmosphere, copied out (either may be NULL). */
int oqg_get_fluxes(oqg_oml *o, double *fnetoc, double *fnetat);

/* ---------------------------------------------------------------------
 * State slots and the adjoint step.  The reference has no adjoint (its model
 * is run forward only); these entry points have no counterpart in it.  They
 * serve gradient computation through the step (reverse mode with
 * checkpoint-every-k recomputation), closed box in FP64 only
 * (OQG_EUNSUPPORTED otherwise).  Slot buffers are device memory the caller
 * owns; copies are queued on the handle's stream.
 * ------------------------------------------------------------------- */

/* Bytes of a full-state slot (p, pm, q, qm, the constraint scalars and the
 * step counter) and of a p-and-q slot.  Either pointer may be NULL. */
int oqg_state_bytes(oqg_handle *h, size_t *full, size_t *pq);
/* Full state to / from a slot: a loaded handle continues bit for bit. */
int oqg_state_save(oqg_handle *h, void *dst);
int oqg_state_load(oqg_handle *h, const void *src);
/* p and q of the current state to a slot: what oqg_adj_step needs of the
 * input state of the step it reverses. */
int oqg_pq_save(oqg_handle *h, void *dst);

/* Sets the adjoint state: the gradient of an objective with respect to the
 * state after the last step, lp, lpm, lq, lqm (nxp, nyp, nl) in host or
 * device memory, NULL for zero; ldpi, ldpip (nl-1) host arrays or NULL.  The
 * accumulated wind adjoint is zeroed.  Makes the adjoint buffers on first use. */
int oqg_adj_set(oqg_handle *h, const double *lp, const double *lpm,
                const double *lq, const double *lqm, const double *ldpi,
                const double *ldpip);
/* Reads the adjoint state and the accumulated gradient with respect to
 * wekp, lwekp (nxp, nyp).  Any pointer may be NULL. */
int oqg_adj_get(oqg_handle *h, double *lp, double *lpm, double *lq,
                double *lqm, double *ldpi, double *ldpip, double *lwekp);
/* Reverses step number step_no (1-based; suppress_comp_mode is transposed
 * when it followed that step, mod(step_no-1, suppress_period) == 0): the
 * adjoint state of the step's output becomes that of its input.  pq is a
 * slot holding p and q of the step's input state (oqg_pq_save).  Queued on
 * the handle's stream; steps are reversed last first. */
int oqg_adj_step(oqg_handle *h, const void *pq, double tdt, long long step_no);
/* One segment of a checkpointed reverse run, queued without host waits:
 * loads the full-state slot ckpt (the state before step first_step_no),
 * recomputes the segment's n steps keeping p and q of each step's input in
 * the slots (n slots of slot_stride bytes from `slots`, device memory), then
 * reverses the n steps last first. */
int oqg_adj_segment(oqg_handle *h, const void *ckpt, void *slots,
                    size_t slot_stride, int n, double tdt,
                    long long first_step_no);
/* The transpose of oqg_set_state applied to the adjoint state: gradients
 * with respect to the p and pm given to oqg_set_state, gp, gpm (nxp, nyp, nl)
 * in host or device memory (either may be NULL). */
int oqg_adj_initial(oqg_handle *h, double *gp, double *gpm);

#ifdef __cplusplus
}
#endif

#endif /* OQG_H */
