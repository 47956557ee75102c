/*
 * libp6cuda -- C ABI of the B200 trial-evaluation backend for Powder 6.
 *
 * Plain pointers and sizes only; no exceptions cross this boundary.  Every
 * function returns a p6_status; on failure p6_last_error() returns a message
 * for the calling thread.  Sessions are opaque, own their device memory and one
 * CUDA stream, and are safe to use from one thread at a time.
 *
 * Reference interfaces replaced (paths inside nitad54448/powder6):
 *   Wyckoff search device layer   js/swarm_wyckoff.js:1293-1720
 *                                 (buffers, dispatchCoords, evaluateCoordsSync,
 *                                  readStateFromGPU, syncStateToGPU) and the
 *                                 kernel swarm_reflection.wgsl:601-1270
 *   Parallel-tempering backend    js/pt_gpu.js:371-423 (RVPTGPU.create / costs /
 *                                 batch / run)
 */
#ifndef P6CUDA_H
#define P6CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes.  The JS/Python host maps every non-OK code to the reference's
 * fallback behaviour (throw -> CPU PT; Wyckoff -> 'wy-error'). */
typedef enum {
  P6_OK = 0,
  P6_ERR_INVALID_ARG = 1,
  P6_ERR_CAPACITY = 2,
  P6_ERR_DEVICE_LOST = 3,
  P6_ERR_TIMEOUT = 4,
  P6_ERR_NOT_CONVERGED = 5,
  P6_ERR_VALIDATION = 6,
  P6_ERR_CUDA = 7
} p6_status;

/* Message of the last failure on this thread ("" when none). */
const char *p6_last_error(void);
/* ABI version, bumped whenever a struct below changes layout. */
int p6_abi_version(void);
/* Host-side fault injection for failure-path tests: after `after_calls` more
 * entry-point calls, return `code` once (0 disables).  Never touches a GPU. */
void p6_debug_inject_failure(int code, int after_calls);

/* ======================================================================== */
/* Wyckoff search                                                            */
/* ======================================================================== */

/* Per-particle Metropolis state, 48 bytes, the layout of ParticleState in
 * swarm_reflection.wgsl:65-87 and SW_STATE_STRIDE (js/swarm_wyckoff.js:45). */
typedef struct {
  float fit;       /* cc - pen * penScale at the scale it was measured */
  float cc;        /* 1 - wR2 */
  float pen;       /* raw penalty, at weight 1 */
  float step_size; /* proposal width, fractional coordinates */
  float temp;      /* rung temperature */
  uint32_t seed;   /* per-chain key of the counter-based generator */
  uint32_t accepted;
  uint32_t pad;
  float best_fit;  /* -1e30: nothing recorded yet */
  float best_cc;
  float best_pen;
  float best_pad;
} p6_wy_particle_state;

/* Static problem description: the packed arrays js/swarm_wyckoff.js:1293-1548
 * uploads, in the reference layouts, plus the kernel constants swInject
 * (js/swarm_wyckoff.js:201-282) compiles in. */
typedef struct {
  int num_particles;
  /* genPack: site | op << 8 | type << 20 | skip << 24, n_assign * n_tot */
  const uint32_t *gen_pack;
  int n_assign;
  int n_tot;
  /* symmetry operators, 12 floats each: r[9] row-major then t[3] */
  const float *sym_packed;
  int n_ops;
  /* per (assignment, site): P[9], T[3]; max_sites is the row stride */
  const float *site_proj;
  int max_sites;
  /* reflections: packed hkl (10 bits each, +512 bias), multiplicity */
  const uint32_t *refl_pack;
  int n_refl;
  /* groups: start, count, Iobs[, weight]; stride 3 or 4 */
  const float *group_meta;
  int n_groups;
  int group_stride;
  /* scattering factors f(s) exp(-B s^2/4), n_refl * n_elem */
  const float *f_tab;
  int n_elem;
  /* restraint table [zByType | rMin (n_elem^2) | rules (7 floats each)] */
  const float *restraint_tables;
  int n_restraint_floats;
  int r_min_off;
  int rule_off;
  int n_rules;
  int max_coord_slots; /* slot capacity (>= the slots the rules claim), <= 256 */
  int geom_slots;      /* == max_coord_slots when any rule has a shape, else 1 */
  /* contact geometry: reduced-basis orth (fractional -> Cartesian) and the
   * integer change of basis, both row-major; inv_orth is Cartesian ->
   * fractional of the cell's own basis (polyhedron moves) */
  double orth[9];
  double xform[9];
  double inv_orth[9];
  int min_image_shell; /* 0 or 1 */
  int count_shell;     /* 0 or 1 */
  int centro;          /* (-I|0) in the group: F is real */
  float pen_clash, pen_bond, pen_coord, pen_geom, poly_prob;
  /* Robbins-Monro step adaptation (exp(a(1-t)), exp(-a t)) and bounds */
  float step_up, step_down, step_min, step_max;
  /* fitness arithmetic: 0 = SFU cosine on the integer-reduced phase,
   * 1 = FMA-pipe polynomial (slower, closer to FP64), 2 = factored FP64:
   * per site and axis cos/sin tables of 2 pi n x built in FP64 from the exact
   * 32-bit turn, |F| as per-reflection monomials of three table entries,
   * FP64 |F|^2 and sums (groups whose rotations are all diagonal: triclinic,
   * monoclinic, orthorhombic; no incremental form; not in batched launches) */
  int cos_mode;
  uint32_t run_key; /* key of the counter-based generator for this session */
  /* per-replica site sums of |F| kept in shared memory so a proposal
   * recomputes only the site it moved (bit-identical results): 1 on; 0 or -1
   * (auto) evaluate every image, which measured faster on the PbSO4 search */
  int incremental;
} p6_wy_problem;

typedef struct p6_wy_session p6_wy_session;

/* Creates the device buffers and uploads the static tables
 * (js/swarm_wyckoff.js:1293-1548).  `device` is a CUDA ordinal. */
p6_status p6_wy_create(const p6_wy_problem *problem, int device, p6_wy_session **out);
/* Frees everything the session owns (the finally of js/swarm_wyckoff.js:2637-2645). */
p6_status p6_wy_destroy(p6_wy_session *s);

/* bufAssign write (js/swarm_wyckoff.js:1767, 2005, 2324). */
p6_status p6_wy_set_assign(p6_wy_session *s, const uint32_t *assign_of);
/* Params.nGroupsActive / penScale (js/swarm_wyckoff.js:2223-2230). */
p6_status p6_wy_set_params(p6_wy_session *s, int n_groups_active, float pen_scale);
/* syncStateToGPU (js/swarm_wyckoff.js:2160-2185): current coordinates
 * (num_particles * max_sites * 3 floats) and per-particle state.  Resets the
 * best-ever half to the current coordinates. */
p6_status p6_wy_sync_state(p6_wy_session *s, const float *positions, const p6_wy_particle_state *state);
/* readStateFromGPU (js/swarm_wyckoff.js:1676-1720): current and best-ever
 * coordinates and the state array.  Any pointer may be NULL. */
p6_status p6_wy_read_state(p6_wy_session *s, float *positions, float *best_positions, p6_wy_particle_state *state);
/* dispatchCoords(coords, isMCMC) (js/swarm_wyckoff.js:1558-1571): one
 * generation for every particle; coords (may be NULL) replaces the current
 * coordinates first.  Asynchronous. */
p6_status p6_wy_dispatch(p6_wy_session *s, const float *coords, int mcmc);
/* evaluateCoordsSync (js/swarm_wyckoff.js:1643-1667): dispatch then read fit
 * (first num_particles floats) and cc (next num_particles floats). */
p6_status p6_wy_evaluate_sync(p6_wy_session *s, const float *coords, int mcmc, float *fit_cc);

/* B200 path: run generations [gen0, gen0 + n_gen) of a schedule entirely on
 * the device.  Each CTA owns one replica ladder (rungs consecutive entries
 * of `ladders`, -1 for an empty rung), so the exchange sweep every
 * `swap_every` generations (js/swarm_wyckoff.js:1825-1851) runs inside the CTA
 * without a host round trip.  sched_groups/sched_pen hold nGroupsActive and
 * penScale per generation (length >= gen0 + n_gen); a change of nGroupsActive
 * re-measures the current state first (js/swarm_wyckoff.js:2226-2256), and
 * reeval_first != 0 does so before generation gen0 as well (the first
 * generation of a restart, or a chunk that starts on a ramp step). */
p6_status p6_wy_set_ladders(p6_wy_session *s, const int32_t *ladders, int n_ladders, int rungs);
p6_status p6_wy_set_schedule(p6_wy_session *s, const int32_t *sched_groups, const float *sched_pen, int n_gen);
p6_status p6_wy_run(p6_wy_session *s, int gen0, int n_gen, int swap_every, int reeval_first);
/* quench (js/swarm_wyckoff.js:2013-2090): with a schedule of step widths set
 * (step_sd[g] for generations g < n_gen), p6_wy_run takes greedy steps --
 * a proposal is kept only if it raises the fitness, the step width is the
 * schedule's, not the adapted one.  step_sd = NULL restores the search. */
p6_status p6_wy_set_quench(p6_wy_session *s, const float *step_sd, int n_gen);
/* Host-buffer form of p6_wy_run: uploads positions/state, runs, reads them back
 * (copies inside the call). */
p6_status p6_wy_run_host(p6_wy_session *s, const float *positions_in, const p6_wy_particle_state *state_in,
                         int gen0, int n_gen, int swap_every, int reeval_first, float *positions_out,
                         float *best_out, p6_wy_particle_state *state_out);

/* Waits for the session's stream, polling with a deadline (P6_ERR_TIMEOUT). */
p6_status p6_wy_synchronize(p6_wy_session *s, double timeout_seconds);
/* Exact coordinate access in the kernel's 32-bit fixed point (x * 2^32). */
p6_status p6_wy_write_positions_fixed(p6_wy_session *s, const uint32_t *current);
p6_status p6_wy_read_positions_fixed(p6_wy_session *s, uint32_t *current, uint32_t *best);
/* Wyckoff-constrained least-squares refinement of coordinates against the
 * grouped |F|^2 of the session's tables (refineCoordinatesAgainstWppf,
 * js/coord_refine.js:266-627): per structure, the closed-form intensity
 * scale, the analytic Jacobian in the constrained space (P^T), Marquardt
 * damping scaled by the diagonal, a trust region of max_step (fractional,
 * infinity norm) and projection back onto the Wyckoff subspaces after each
 * step.  The group intensities, derivatives and normal equations are FP64 on
 * the device (one CTA per structure); the damping control runs on the host
 * for all structures in lock step.  coords (n * max_sites * 3, fractional) are
 * refined in place; r_start / r_final are the weighted wR(F^2), chi2 the
 * final weighted residual, iterations the accepted steps.  NULL opts: the
 * reference's defaults (60 iterations, lambda 1e-3 x10 / x0.4 up to 1e8,
 * tol_step 1e-6, tol_chi 1e-9, max_step 0.05).  Any output may be NULL. */
typedef struct {
  int max_iter;
  double lambda0, lambda_up, lambda_down, lambda_max, tol_step, tol_chi, max_step;
} p6_wy_refine_opts;
p6_status p6_wy_refine(p6_wy_session *s, int n, const uint32_t *assign, double *coords,
                       const p6_wy_refine_opts *opts, double *r_start, double *r_final, double *chi2,
                       int *iterations, int *converged);
/* Launch shape of the fused search (p6_wy_run): each replica ladder of 8 on
 * one CTA of 8 warps (1) or on a thread-block cluster of two 4-warp CTAs (2,
 * the default; clash-penalty problems with staged tables and the full
 * evaluation only, others use 1).  Two CTAs per
 * ladder spread the ladders evenly over the SMs; the results are the same
 * bit for bit.  The reference runs one workgroup per replica. */
p6_status p6_wy_set_ladder_split(p6_wy_session *s, int ctas_per_ladder);
/* syncStateToGPU after a prune (js/swarm_wyckoff.js:2303-2336): current and
 * best coordinates in fixed point and the particle states, written together
 * so the chains that keep their assignment keep their best structure exactly. */
p6_status p6_wy_write_state_fixed(p6_wy_session *s, const uint32_t *current, const uint32_t *best,
                                  const p6_wy_particle_state *state);
/* Parity support: record, for the next dispatch, each particle's proposal
 * (max_sites * 3 fixed-point words) and a record of 8 floats
 * {f_new, cc, pen_scaled, u, accepted, f_old, temp, step_before}. */
p6_status p6_wy_set_trace(p6_wy_session *s, int enable);
p6_status p6_wy_read_trace(p6_wy_session *s, uint32_t *proposals, float *records);
/* mult * |F|^2 of every reflection of each particle's last traced evaluation
 * (num_particles * n_refl floats; reflections past the active groups untouched). */
p6_status p6_wy_read_trace_ic(p6_wy_session *s, float *ic);
/* A rigid fragment with torsions (the config-5 molecule): the sites of the
 * session's single assignment are the fragment's atoms in order, and each
 * replica searches a translation t (fractional), a unit quaternion q and the
 * torsion angles instead of the sites' coordinates.  Atom i = t + to_frac .
 * R(q) . (ref_i after the torsions, applied in order, each turning the atoms of
 * `moving[k]` about the bond axis_b[k] -> axis_c[k] by its angle).  A
 * proposal moves every parameter (p = 1/4) or one group: the translation
 * (steps of width x trans_step), the orientation (a turn of width x
 * angle_step radians about a random axis) or one torsion (width x
 * angle_step); the structure-factor fitness, penalty and acceptance are the
 * search's own.  The reference searches molecules as sites held by distance
 * rules (js/molecule_rules.js:1-18, swarm_reflection.wgsl:893-1130); this is
 * the direct-space parametrisation of the same molecule.  NULL turns it off. */
typedef struct {
  int n_atoms;          /* <= 32 and <= max_sites */
  int n_tors;           /* <= 8 */
  int axis_b[8], axis_c[8];
  uint32_t moving[8];   /* bit i: atom i turns with torsion k */
  double ref_xyz[96];   /* reference geometry, Cartesian A about its centroid */
  double to_frac[9];    /* Cartesian -> fractional of the cell, row-major */
  double trans_step, angle_step;
} p6_wy_fragment;
p6_status p6_wy_set_fragment(p6_wy_session *s, const p6_wy_fragment *fragment);
/* Per particle 16 floats: t[3], q[4] (w, x, y, z), the torsion angles; the
 * write sets the current and the best parameters, the read returns both. */
p6_status p6_wy_write_fragment_state(p6_wy_session *s, const float *current);
p6_status p6_wy_read_fragment_state(p6_wy_session *s, float *current, float *best);
/* Parity support: the fixed-point coordinates (n_atoms * 3 words per vector)
 * of n parameter vectors, mapped on the device as the search maps them. */
p6_status p6_wy_debug_fragment(p6_wy_session *s, const float *params, int n, uint32_t *coords);
/* The FP64 fitness sums {sum w Ic^2, sum w Io^2, sum w Ic Io} over the active
 * groups of each particle's last traced evaluation (num_particles * 3
 * doubles); cc = sco / sqrt(scc soo), the grouped wR2^2 after the best scale
 * is 1 - cc^2 (js/swarm_wyckoff.js:679-766). */
p6_status p6_wy_read_trace_sums(p6_wy_session *s, double *sums);
/* The generated cell of one particle's current coordinates, in genPack order,
 * fixed point (n_tot * 3 words). */
p6_status p6_wy_debug_expand(p6_wy_session *s, int particle, uint32_t *atoms);
/* Milliseconds of the last p6_wy_run / p6_wy_dispatch kernel (CUDA events on
 * the session stream). */
p6_status p6_wy_last_kernel_ms(p6_wy_session *s, float *ms);
/* Session layout: whether site sums are incremental, shared memory per CTA,
 * and the resident grid (any pointer may be NULL). */
p6_status p6_wy_query(p6_wy_session *s, int *incremental, int *smem_bytes, int *max_grid);
/* Kernel launches made by this session so far. */
p6_status p6_wy_launch_count(p6_wy_session *s, long long *count);


/* ======================================================================== */
/* Parallel tempering (Rietveld)                                             */
/* ======================================================================== */

/* One phase and one dataset, X-rays, TCH profile: the arrays RVPTGPU.compile
 * packs (js/pt_gpu.js:20-227) in plain form.  The full parameter vector is
 * [scale, a, b, c, alpha, beta, gamma, U, V, W, X, Y, zero, Biso, bkg0, ...]
 * (GSAS units for U..Y); `index` maps the nv refined parameters into it, and
 * lo/hi/scales are ctx.info[j].lo/hi and ctx.setup.scales
 * (js/rietveld_core.js:2147-2170). */
typedef struct {
  int n_refl;              /* reflections over the cell envelope (generateReflections, :247-276) */
  const int32_t *hkl;      /* 3 per reflection */
  const int32_t *mult;
  int n_reps;              /* coset representatives modulo centring (cosets, :164-180) */
  const int32_t *rep_rot;  /* 9 per representative, row-major */
  const double *rep_trans; /* 3 per representative */
  int n_atoms;
  const double *atom_pos;  /* 3 per atom, fractional */
  const double *atom_wmult;/* site multiplicity / n_reps */
  const double *atom_occ;
  const double *ff_a, *ff_b, *ff_c; /* 5, 5, 1 per atom: f0(s) = c + sum a exp(-b (s/2)^2) */
  int n_points;
  const double *tth;       /* ascending */
  const double *y, *w;
  double lambda1, lambda2, ratio, pol_k, min_fwhm, dmin;
  int n_bkg;               /* Chebyshev terms */
  int n_full;
  const double *full_values;
  int nv;
  const int32_t *index;
  const double *lo, *hi, *scales;
  int cubic;               /* b = c = a */
  int chains;
  double max_temp;
  uint32_t seed;
  /* March-Dollase preferred orientation (js/rietveld_core.js:824-853, GPU
   * js/pt_gpu.js:159-160).  has_po = 0: off (factor 1).  Otherwise the March
   * parameter r is full_values[n_bkg + 14] (the entry after the background),
   * the direction po_dir is a reciprocal-lattice vector, and the factor of
   * reflection k averages (r^2 cos^2 a + sin^2 a / r)^(-3/2) over its
   * equivalents eq_hkl[3 * eq_start[k] .. 3 * eq_start[k + 1]), a = the angle
   * between the equivalent and po_dir in the current reciprocal metric
   * (r <= 0 or |r - 1| < 1e-12: factor 1). */
  int has_po;
  const int32_t *eq_start; /* n_refl + 1 */
  const int32_t *eq_hkl;   /* 3 per equivalent */
  double po_dir[3];
  /* SL/HL axial-divergence asymmetry of the TCH profile (js/profile.js:608-617,
   * :686-722, :737-740, area correction :799-826; GPU js/pt_gpu.js:332-353).
   * has_asym = 0: symmetric.  Otherwise SL and HL are the two full-vector
   * entries after the background (and after r when has_po); each peak gets
   * asym = SL / tan(theta) + HL, a doubled window and the area correction. */
  int has_asym;
  /* Fit method (js/pt_gpu.js:259-297): 0 Rietveld (heights from the
   * structure); 1 WPPF / Le Bail: every reflection's height is free and
   * non-negative, solved in every evaluation by NNLS against the observed
   * pattern minus the background (atoms unused, n_atoms may be 0; at most 64
   * envelope reflections). */
  int method;
  /* Sample displacement and transparency (js/pt_gpu.js:169-171, :355): when
   * set, the two full-vector entries after SL, HL (or after 'po', or after
   * the background) are disp and transp, and every peak moves by
   * (-disp 1e-3 cos(theta) + transp sin(2 theta)) degrees before the zero
   * point. */
  int has_shift;
} p6_pt_problem;

typedef struct p6_pt_session p6_pt_session;

/* RVPTGPU.create (js/pt_gpu.js:371-406): device buffers for the plan. */
p6_status p6_pt_create(const p6_pt_problem *problem, int device, p6_pt_session **out);
p6_status p6_pt_destroy(p6_pt_session *s);
/* create().costs (js/pt_gpu.js:402): chi^2 of n_vectors refined-parameter
 * vectors (nv each); ycalc (may be NULL) receives n_vectors * n_points floats. */
p6_status p6_pt_costs(p6_pt_session *s, const double *vectors, int n_vectors, double *costs, float *ycalc);
/* create().initial (js/pt_gpu.js:400): chain c starts from vectors[c % n]. */
p6_status p6_pt_initial(p6_pt_session *s, const double *vectors, int n_vectors);
/* create().batch (js/pt_gpu.js:403): `count` sweeps of nv proposals per
 * chain with even/odd exchanges, or one evaluation of the start (bootstrap).
 * Asynchronous; read the state to wait. */
p6_status p6_pt_batch(p6_pt_session *s, int count, int bootstrap);
/* State after the last batch: `state` in the reference layout
 * (chains x (3 nv + 12) floats: x, proposal, best, cost, bestCost, sweep,
 * accepted, proposals, swaps, swapAttempts, valid, log u, unsolved,
 * proposalCost, feasible), and exactly: x, best (chains x nv doubles),
 * costs (cost, bestCost per chain), counters (accepted, proposals, swaps,
 * swapAttempts per chain).  Any pointer may be NULL. */
p6_status p6_pt_read_state(p6_pt_session *s, float *state, double *x, double *best, double *costs, double *counters);
p6_status p6_pt_synchronize(p6_pt_session *s, double timeout_seconds);
p6_status p6_pt_last_batch_ms(p6_pt_session *s, float *ms);
/* Parity support: record, for every chain, the decisions of the last sweep
 * of each p6_pt_batch: {exchange tried, swapped, la, log u} and then per
 * move {parameter index, proposed value, log u, cost before, proposal cost,
 * accepted} (chains * (4 + 6 nv) doubles), for replaying the Metropolis and
 * exchange rules of temper (js/rietveld_core.js:2171-2241) on the host. */
p6_status p6_pt_set_trace(p6_pt_session *s, int enable);
p6_status p6_pt_read_trace(p6_pt_session *s, double *out);
p6_status p6_pt_launch_count(p6_pt_session *s, long long *count);
/* CTAs per chain in the sweeps: 2 runs each chain on a two-CTA cluster (the
 * pattern's tiles split between them, chi^2 combined through distributed
 * shared memory), chosen at creation when twice the chains fit the SMs;
 * 1 is one CTA per chain.  Trajectories differ between the two only by the
 * order of the chi^2 sum. */
p6_status p6_pt_set_split(p6_pt_session *s, int ctas_per_chain);
p6_status p6_pt_get_split(p6_pt_session *s, int *ctas_per_chain);

/* Least-squares finish after tempering (js/rietveld_core.js:1953-2140), in
 * FP64 on the device: patterns, the finite-difference Jacobian (fdStep
 * :526-538, central where defaultLimits :486-508 allow), the normal
 * equations and the damped Cholesky solve (solveSPD :1304-1335).
 *
 * p6_pt_model_costs: chi^2 of n refined vectors (n x nv) with the FP64 model
 *   (the re-score of new per-chain bests, js/pt_gpu.js:419-421).
 * p6_pt_normal: A = J'WJ (nv x nv, row-major), g = J'W r, f = chi^2 at x.
 * p6_pt_linear_start: one Gauss-Newton step on the scale and background
 *   parameters from x, kept if it lowers chi^2 (:2252-2263); chi2 may be NULL.
 * p6_pt_lm: lm() from x (in/out) within the session's bounds, at most
 *   max_iter iterations, relative chi^2 tolerance tol (<= 0: 1e-5).
 *   out (may be NULL): chi^2, iterations, accepted steps, exit code
 *   (0 iteration limit, 1 chi^2 change below tol, 2 projected gradient below
 *   tolerance, 3 singular system, 4 stalled, 5 all parameters at limits,
 *   6 stopped at the Gaussian-variance limit). */
p6_status p6_pt_model_costs(p6_pt_session *s, const double *x, int n, double *chi2);
p6_status p6_pt_normal(p6_pt_session *s, const double *x, double *A, double *g, double *f);
p6_status p6_pt_linear_start(p6_pt_session *s, double *x, double *chi2);
p6_status p6_pt_lm(p6_pt_session *s, double *x, int max_iter, double tol, double *out);

/* p6_pt_costs without any device allocation.  No reference counterpart: the
 * WebGPU backend has no caller that must avoid allocating.
 *
 * Same arguments, kernel and results as p6_pt_costs, but the scratch (the
 * uploaded vectors, the costs and the optional patterns) lives in one
 * file-scope device array of P6_PT_STATIC_SCRATCH_BYTES per device instead of
 * buffers that p6_pt_costs grows with cudaMalloc.  For callers that cannot
 * allocate: cudaMalloc/cudaFree synchronise the whole device, which stalls a
 * host that keeps tempering sweeps in flight on other streams while it
 * validates probe costs, and a host that has handed all free HBM to its own
 * pool has nothing left for a lazy allocation to take.
 *
 * Limit: align256(n_vectors * nv * 8) + align256(n_vectors * 8)
 * + (ycalc ? n_vectors * n_points * 4 : 0) <= P6_PT_STATIC_SCRATCH_BYTES;
 * larger requests return P6_ERR_CAPACITY (split them, or use p6_pt_costs).
 * Nothing in the scratch has to start at zero: each call writes every byte it
 * reads.  All sessions on a device share the one array, so calls that overlap
 * in time (two host threads, on the same or different sessions) race; a
 * single thread never overlaps itself because the call returns only after its
 * stream has finished.  The first call on each device looks up the array's
 * address (cudaGetSymbolAddress); make that first call outside any stream
 * capture.  The address is looked up again when the device's context has
 * changed since (cudaDeviceReset replaces the context and reloads the
 * module), so the first call after a reset must also come outside a capture.
 * The call waits for its stream at most P6_PT_STATIC_WAIT_SECONDS and then
 * returns P6_ERR_TIMEOUT with its copies possibly still in flight: call
 * p6_pt_synchronize before reusing or freeing `costs` and `ycalc`. */
#define P6_PT_STATIC_SCRATCH_BYTES (4u << 20)
#define P6_PT_STATIC_WAIT_SECONDS 60.0
p6_status p6_pt_costs_static(p6_pt_session *s, const double *vectors, int n_vectors, double *costs, float *ycalc);

/* How many vectors the session's allocating scratch (grown by p6_pt_costs
 * with cudaMalloc) holds now; 0 until p6_pt_costs first runs.  Lets a caller
 * check that it only ever used the allocation-free call. */
p6_status p6_pt_vector_capacity(p6_pt_session *s, int *n_vectors);

/* Many searches in one persistent launch.  The sessions (same device and
 * cos_mode, incremental evaluation off, at most 8 rungs, ladders and
 * schedules set) keep their own tables and state; the batch runs all their
 * ladders in one launch of persistent CTAs that take (search, ladder) items
 * from a list -- longest estimated ladder first (order 0) or in search order
 * (1) -- each CTA staging the tables of the search it is working on.  The
 * dynamic shared memory of the launch is the largest search's.  No
 * reference counterpart: the reference runs one search per worker
 * (js/wyckoff_worker.js); each search's results are those of p6_wy_run. */
typedef struct p6_wy_batch p6_wy_batch;
p6_status p6_wy_batch_create(p6_wy_session *const *sessions, int n_sessions, p6_wy_batch **out);
p6_status p6_wy_batch_destroy(p6_wy_batch *b);
/* Launch shape: ctas_per_sm persistent CTAs per SM (0: the occupancy limit,
 * at most the value p6_wy_batch_query reports) and the item order. */
p6_status p6_wy_batch_set_launch(p6_wy_batch *b, int ctas_per_sm, int order);
p6_status p6_wy_batch_query(p6_wy_batch *b, int *max_ctas_per_sm, int *smem_bytes, int *n_items, long long *launches);
/* Generations [gen0[i], gen0[i] + n_gen[i]) of session i, exchange every
 * swap_every generations; use_graph != 0 replays the launch from a CUDA
 * graph captured on first use.  Asynchronous; the sessions' later calls
 * wait for it. */
p6_status p6_wy_batch_run(p6_wy_batch *b, const int32_t *gen0, const int32_t *n_gen, int swap_every, int reeval_first,
                          int use_graph);
p6_status p6_wy_batch_synchronize(p6_wy_batch *b, double timeout_seconds);
p6_status p6_wy_batch_last_ms(p6_wy_batch *b, float *ms);

/* ======================================================================== */
/* Proposal network (learned search)                                         */
/* ======================================================================== */

/* A 3-layer MLP, d_in -> width -> width -> d_out with ReLU, trained on the
 * GPU (FP32 master weights, Adam, masked mean-squared error with 0/1 masks)
 * and evaluated with bf16 copies of its weights.  No reference counterpart:
 * the reference's proposals are all random (swarm_reflection.wgsl:657-725).
 * Parameters flatten as W1 (d_in x width, row-major), b1, W2, b2, W3
 * (width x d_out), b3.  Host arrays: X rows x d_in, T and mask rows x d_out. */
typedef struct p6_mlp p6_mlp;
p6_status p6_mlp_create(int d_in, int width, int d_out, uint32_t seed, int device, p6_mlp **out);
p6_status p6_mlp_destroy(p6_mlp *n);
/* One generation of a learned search on session s: K candidate proposals
 * per replica (the plain search's move distribution, with a 64-feature
 * description each), the network's first output as the predicted fitness
 * gain, the best-ranked candidate evaluated with the exact fitness and the
 * usual Metropolis test (K = 1, net = NULL: the plain move, no network).
 * Optional host outputs per replica: the chosen candidate's features
 * (num_particles x 64), the evaluated fitness change f_new - f_old, whether
 * it was accepted (0/1), and the predicted gain.  The network's scratch is
 * used on the session's stream: do not train it meanwhile. */
p6_status p6_wy_learned_step(p6_wy_session *s, p6_mlp *net, int K, int gen, int swap_every, int reeval_first,
                             float *features, float *gains, float *accepted, float *scores);
/* Marks the start (end = 0) or the end (end = 1) of a span on the session's
 * stream, for p6_wy_last_kernel_ms (the device time of a multi-launch loop). */
p6_status p6_wy_time_mark(p6_wy_session *s, int end);
/* Copies the FP32 parameters out (get) and/or in (set); count receives their number. */
p6_status p6_mlp_params(p6_mlp *n, float *get, const float *set, long long *count);
/* Gradient of the loss over the given rows (flat, like the parameters) and the loss. */
p6_status p6_mlp_gradients(p6_mlp *n, const float *X, const float *T, const float *mask, int rows, float *grad,
                           float *loss);
/* `epochs` passes of Adam over shuffled minibatches; epoch_loss (may be NULL) gets the mean loss of each. */
p6_status p6_mlp_train(p6_mlp *n, const float *X, const float *T, const float *mask, int rows, int epochs, int batch,
                       float lr, uint32_t seed, float *epoch_loss);
/* Inference with the bf16 weights: Y (rows x d_out). */
p6_status p6_mlp_predict(p6_mlp *n, const float *X, int rows, float *Y);

/* ======================================================================== */
/* Profile contraction with the cell and profile fixed                       */
/* ======================================================================== */

/* With the cell and profile fixed, the calculated patterns of all replicas
 * are Y = I . P: intensities I (replicas x reflections, the per-reflection
 * heights mult Lp |F|^2 / area each replica's structure gives, as
 * js/rietveld_core.js:881-886 forms them) times the banded profile matrix P
 * (reflections x points, the unit-height Ka1 + Ka2 columns of
 * js/profile.js:1013-1090).  The reference renders every trial pattern peak
 * by peak; here the product runs on the tensor cores (split-BF16, FP32
 * accumulation) or on the CUDA cores in FP32, and the weighted chi^2 of each
 * replica against the observed pattern is reduced in FP64. */
typedef struct {
  int n_refl;              /* K: reflections, sorted by 2-theta */
  int n_points;            /* N: pattern points */
  int max_replicas;        /* M capacity */
  const float *profile_t;  /* P transposed: n_points x n_refl, row j = the profile values at point j */
  const float *yobs;       /* n_points observed counts */
  const float *w;          /* n_points weights (w <= 0 excludes a point) */
} p6_ct_problem;

/* P6_CT_SPLIT3_BF16: three bf16 parts per operand (exact to 2^-27) and six
 * products, so the tensor core's FP32 accumulation is what is left (chi^2
 * within about 4e-6 of FP64 against 1.2e-5 for the two-part split); twice
 * the MMA work of P6_CT_SPLIT_BF16. */
/* P6_CT_FP32_DENSE: the FP32 CUDA-core product over every reflection at
 * every point, the dense render js/pt_gpu.js:249-252 (`columns`, `targets`)
 * performs; P6_CT_FP32 runs the same product over each tile's band only. */
enum { P6_CT_SPLIT_BF16 = 0, P6_CT_FP32 = 1, P6_CT_SPLIT3_BF16 = 2, P6_CT_FP32_DENSE = 3 };

typedef struct p6_ct_session p6_ct_session;

p6_status p6_ct_create(const p6_ct_problem *problem, int device, p6_ct_session **out);
p6_status p6_ct_destroy(p6_ct_session *s);
/* Uploads I (n_replicas x n_refl, row-major, host memory). */
p6_status p6_ct_set_intensities(p6_ct_session *s, const float *intensities, int n_replicas);
/* Asynchronous: Y = I . P with `method` and chi^2 per replica; store_pattern
 * != 0 also keeps Y (n_replicas x n_points) on the device. */
p6_status p6_ct_evaluate(p6_ct_session *s, int method, int store_pattern);
/* Waits, then copies chi^2 (n_replicas doubles) and, if stored and
 * requested, Y.  Either pointer may be NULL. */
p6_status p6_ct_read(p6_ct_session *s, double *chi2, float *pattern);
/* Upload, evaluate, read chi^2: the end-to-end call. */
p6_status p6_ct_run_host(p6_ct_session *s, const float *intensities, int n_replicas, int method, double *chi2);
p6_status p6_ct_synchronize(p6_ct_session *s);
/* Device time of the last p6_ct_evaluate. */
p6_status p6_ct_last_ms(p6_ct_session *s, float *ms);
/* Band statistics: K-blocks (64 reflections) summed over the 256-point tiles
 * the tensor-core path runs, reflections summed over the 128-point tiles of
 * the FP32 path, the number of 256-point tiles, kernels launched. */
/* Fitted scale (fitted != 0): chi^2 of each replica at its best scale,
 * min over s >= 0 of sum w (y - s Y)^2 = sum w y^2 - a^2 / b with a = sum
 * w y Y and b = sum w Y^2 (FP64 sums), as a structure search with the scale
 * free needs; fitted == 0 (the default) takes the intensities as scaled. */
p6_status p6_ct_set_fitted(p6_ct_session *s, int fitted);
/* Waits, then copies the fitted scales of the last evaluation (n_replicas doubles). */
p6_status p6_ct_read_scale(p6_ct_session *s, double *scale);
p6_status p6_ct_query(p6_ct_session *s, long long *band_kblocks, long long *band_cols128, int *n_tiles,
                      long long *launches);

/* Fixed-profile fitness in Gram form, for every later evaluation of the
 * session (p6_wy_run, p6_wy_dispatch, ...): with the cell and profile fixed,
 * y_calc = s I . P with I = mult |F|^2 per reflection, and the weighted
 * chi^2 at the best scale is sum w y^2 - a^2 / b with a = v . I and
 * b = I G I^T, where v = P (w y) and G = P W P^T (banded, symmetric) are
 * fixed.  The search kernel forms a and b from its FP64 intensities, so the
 * fitness cc becomes 1 - Rwp (exact in FP64, no pattern formed) and the
 * whole search stays one launch (also in p6_wy_batch_run, each session
 * with its own pattern).  v: n_refl doubles; band: the upper band of G by
 * diagonal, band[d * n_refl + k] = G[k][k + d] (0 past the end), d = 0..bw;
 * syy = sum w y^2.  In cos mode 2 the intensities are FP64, in modes 0 and
 * 1 FP32; a and b are summed in FP64 either way.  Every reflection is
 * evaluated (the resolution part of the schedule is not used).  v == NULL
 * returns to the grouped-intensity fitness. */
p6_status p6_wy_set_profile(p6_wy_session *s, const double *v, const double *band, int bw, double syy);

/* Fixed-profile Wyckoff search: the search of p6_wy_run with the profile
 * chi^2 as its energy, for a cell and profile held fixed.  The contraction
 * session's reflections must be the search session's (same count and order,
 * profile columns carrying Lp and the peak shape, so a row of intensities is
 * mult |F|^2 per reflection) and hold at least as many replicas.  Per
 * generation, on the search session's stream: the search kernel proposes a
 * move for every replica and writes the proposal's intensities into the
 * contraction's buffer; Y = I . P runs with `method` (P6_CT_*) and gives the
 * chi^2 at each replica's best scale over the first n_active_points points
 * (<= 0: all); an acceptance kernel applies the Metropolis test with the
 * replica's fitness 1 - Rwp - penalty, keeps the best structures, adapts the
 * step and exchanges replicas along the ladders every swap_every
 * generations.  Every reflection is evaluated (the resolution part of the
 * schedule is not used); the penalty scale and the quench follow the
 * session's schedules.  init != 0 first evaluates the current structures at
 * generation gen0 and makes them the chains' energies (n_gen may then be 0).
 * A rigid-fragment session (p6_wy_set_fragment) runs too: a proposal's
 * fragment parameters follow its coordinates through the acceptance, the
 * bests and the exchange.
 * Asynchronous: p6_wy_synchronize waits and also reports a contraction wait
 * that ran out.  In the particle states, cc holds 1 - Rwp. */
p6_status p6_wy_profile_run(p6_wy_session *s, p6_ct_session *ct, int method, int gen0, int n_gen, int swap_every,
                            int init, int n_active_points);

/* ======================================================================== */
/* Dual-space charge flipping on a powder reflection model                   */
/* ======================================================================== */
/* The cycle of charge_flipping.wgsl:182-632 in the order
 * js/charge_flipping_worker.js:2353-2395 dispatches it: F -> rho (inverse
 * 3-D FFT, 1/n^3), the flip threshold delta = delta_sigma * sigma(Re rho),
 * the flip (Re rho < delta -> -Re rho, Im rho = 0), rho -> F, the R factor on
 * cluster totals, the Le Bail repartition of each cluster's observed
 * intensity, the space-group symmetrisation damped by sym_lambda, the
 * amplitude constraint (a quarter-turn for weak orbits), hard zeros on the
 * absent reflections and F(000), and the best iterate kept on the device.
 * Independent trials (random starts and settings of one model) run in the
 * same launches.  Grids are interleaved complex floats, index h + k n + l n^2
 * with the Miller indices wrapped into 0..n-1. */
typedef struct {
  int n;                               /* grid edge: 8, 16, 32, 64 or 128 */
  int n_orbits;
  const uint32_t *orbit_start;         /* n_orbits: first member of each orbit */
  const uint32_t *orbit_count;         /* n_orbits: members of each orbit */
  int n_members;
  const uint32_t *orbit_idx;           /* n_members: grid index, | 0x80000000 when the member stores the Friedel mate */
  const float *phase;                  /* 2 n_members: exp(+2 pi i h0.t) of the operator that produced the member */
  int n_clusters;
  const uint32_t *cluster_orbit_start; /* n_clusters: first orbit (the orbits of a cluster are consecutive) */
  const uint32_t *cluster_n_orbits;    /* n_clusters */
  const float *cluster_obs_i;          /* n_clusters: observed intensity of the cluster */
  int n_absent;
  const uint32_t *absent_idx;          /* n_absent: grid indices held at zero */
} p6_cf_model;

typedef struct {
  float delta_sigma;                   /* flip threshold in units of the map's sigma */
  float sym_lambda;                    /* 0: P1 charge flipping .. 1: strict space-group symmetry */
  uint32_t seed;                       /* phase restarts of reflections whose amplitude collapsed */
  const uint8_t *weak;                 /* n_orbits flags (quarter-turn instead of the amplitude constraint), or NULL */
} p6_cf_trial;

typedef struct p6_cf_session p6_cf_session;

/* Replaces the GPU setup of runChargeFlippingGPU (js/charge_flipping_worker.js:1997-2330). */
p6_status p6_cf_create(const p6_cf_model *model, int n_trials, const p6_cf_trial *trials, int device,
                       p6_cf_session **out);
p6_status p6_cf_destroy(p6_cf_session *s);
/* Uploads the starting F grid (2 n^3 floats) of one trial, or of every trial
 * when trial < 0, makes it the best iterate and resets the best R to +inf. */
p6_status p6_cf_set_grid(p6_cf_session *s, int trial, const float *grid);
/* Runs `cycles` cycles of every trial (the loop of
 * js/charge_flipping_worker.js:2353-2395); r_history (n_trials x cycles, row
 * per trial, may be NULL) receives the R factor of each cycle.  Blocking. */
p6_status p6_cf_run(p6_cf_session *s, int cycles, float *r_history);
/* Best R of every trial (n_trials floats). */
p6_status p6_cf_best_r(p6_cf_session *s, float *best_r);
/* which = 0: the current F grid (2 n^3 floats); 1: the best F grid; 2: the
 * density of the best grid (n^3 floats, the real part of its inverse
 * transform with 1/n^3). */
p6_status p6_cf_read(p6_cf_session *s, int trial, int which, float *out);
/* Device time of the last p6_cf_run, and the kernels launched so far. */
p6_status p6_cf_last_ms(p6_cf_session *s, float *ms);
p6_status p6_cf_launch_count(p6_cf_session *s, long long *count);
/* Runs `cycles` cycles as separate launches with events between them and
 * returns the mean device time of one transform pass (one axis, every trial,
 * all chunks) and of one reciprocal step; the R factors of these cycles are
 * not kept. */
p6_status p6_cf_time_kernels(p6_cf_session *s, int cycles, float *fft_pass_ms, float *reciprocal_ms);

/* Philox4x32-10 of one (counter, key) on the device: known-answer check. */
p6_status p6_philox_device(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif

#endif /* P6CUDA_H */
