/*
 * gemsgpu.h -- C ABI of the B200 (sm_100a) force/neighbour path of GEMS.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes.  A
 * Fortran `bind(C)` interface module binds these names directly (see the
 * integration notes shipped with this library).  Every entry point replaces
 * one reference routine or plug point, cited as file:line within
 * alexispaz/GEMS.
 *
 * Units are GEMS internal units (Angstrom, uma, ps; energy uma*A^2/ps^2)
 * unless a function says eV.  Per-atom vectors use the GEMS interleaved
 * layout [x1, y1, z1, x2, ...] of group_switch_vectorial
 * (src/Groups.F90:553-585).  The library owns all device memory; the caller
 * owns host buffers, which are copied and never retained past a call.
 *
 * Status codes: 0 on success, a negative GEMSGPU_ERR_* otherwise; the text of
 * the last error of a context is returned by gemsgpu_last_error.  No entry
 * point aborts, traps or exits the process.
 *
 * Threading: one host thread per context at a time; every context owns one
 * CUDA stream and all of its work is ordered on that stream.
 */
#ifndef GEMSGPU_H
#define GEMSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GEMSGPU_OK 0
#define GEMSGPU_ERR_ARG (-1)      /* bad argument / unknown handle          */
#define GEMSGPU_ERR_OOM (-2)      /* device allocation failed               */
#define GEMSGPU_ERR_CUDA (-3)     /* CUDA runtime error                      */
#define GEMSGPU_ERR_OVERFLOW (-4) /* neighbour capacity exceeded, not healed */
#define GEMSGPU_ERR_LOST (-5)     /* atom outside the cell grid of a box     */
#define GEMSGPU_ERR_NAN (-6)      /* non-finite position or force            */
#define GEMSGPU_ERR_STATE (-7)    /* call out of order (no force field, ...) */
#define GEMSGPU_ERR_TIMEOUT (-8)  /* bounded device wait expired             */
#define GEMSGPU_ERR_NODEV (-9)    /* no usable CUDA device                   */
#define GEMSGPU_ERR_FULL (-10)    /* arena has no room for the request       */

/* force-field kinds (the `interact ... under <pot>` keywords) */
#define GEMSGPU_FF_NONE 0
#define GEMSGPU_FF_LJ 1      /* lj / plj, Pairs.F90:198-370      */
#define GEMSGPU_FF_SMATB 2   /* tb, TB.F90:106-586               */
#define GEMSGPU_FF_TERSOFF 3 /* tersoff, Tersoff.f90:131-341     */

/* integrators (the `evolve <alg>` keywords) */
#define GEMSGPU_INT_NONE 0
#define GEMSGPU_INT_VV 1    /* v_verlet, Integration.F90:1150-1186 */
#define GEMSGPU_INT_ERMAK 2 /* ermak, Integration.F90:909-1031     */
#define GEMSGPU_INT_FIRE 3  /* fire, FIRE.f90:40-141 (intent)      */

/* arithmetic of the force kernels */
#define GEMSGPU_PREC_FP64 0  /* plain FP64: the drop-in                  */
#define GEMSGPU_PREC_MIXED 1 /* FP32 pair math, FP64 accumulation        */

typedef struct gemsgpu_ctx gemsgpu_ctx;
typedef struct gemsgpu_pool gemsgpu_pool;
typedef struct gemsgpu_server gemsgpu_server;

/* a job of the serving loop: one free SMA-TB cluster */
#define GEMSGPU_JOB_FIRE 0   /* relax with FIRE to max|F| < fmax, <= steps iterations */
#define GEMSGPU_JOB_MD 1     /* `steps` Ermak steps at temp (rounded up to whole chunks) */
#define GEMSGPU_JOB_QUEUED 0
#define GEMSGPU_JOB_RUNNING 1
#define GEMSGPU_JOB_DONE 2
#define GEMSGPU_JOB_FAILED 3
typedef struct gemsgpu_job {
  int natoms;
  const double* pos;   /* 3 natoms, copied at submit */
  double mass;         /* uma */
  double smatb[7];     /* A, xi, p, q, r0, rci, rce as gemsgpu_set_smatb */
  int kind;            /* GEMSGPU_JOB_FIRE or GEMSGPU_JOB_MD */
  int steps;
  double dt;           /* ps; FIRE: initial dt, dt_max = 10 dt */
  double temp, gamma;  /* MD: Ermak bath */
  double fmax;         /* FIRE: convergence, eV/A */
  uint64_t seed;       /* MD: Philox stream */
} gemsgpu_job;

/* ------------------------------------------------------------ context */

/* Create a context on CUDA device `device`.  max_atoms / max_systems size
 * the HBM arena (0 = grow on demand). */
int gemsgpu_create(int device, int64_t max_atoms, int max_systems,
                   gemsgpu_ctx** out);
int gemsgpu_destroy(gemsgpu_ctx* ctx);
/* Copy the last error message of ctx (NUL-terminated) into buf. */
int gemsgpu_last_error(gemsgpu_ctx* ctx, char* buf, int len);
/* Library version string (static storage). */
const char* gemsgpu_version(void);

/* ------------------------------------------------------------ systems */

/* A system is one GEMS group with its interaction group(s) and integrator.
 * Replaces the intergroup constructor (src/Neighbour.F90:255-295) and the
 * atom arrays of group_switch_vectorial (src/Groups.F90:553-585). */
int gemsgpu_system_create(gemsgpu_ctx* ctx, int natoms, int ntypes, int* sys);
int gemsgpu_system_destroy(gemsgpu_ctx* ctx, int sys);

/* Copy positions (3n), velocities (3n, may be NULL = zero), masses (n) and
 * 0-based types (n, may be NULL = all 0) to the device.  Masses follow
 * set_mass (src/Set_Properties.f90:168-191).  acel is reset to zero, as for
 * freshly created atoms (src/Atoms.F90:184). */
int gemsgpu_upload(gemsgpu_ctx* ctx, int sys, const double* pos,
                   const double* vel, const double* mass, const int* type);
/* Replace positions only (dinamic_from_xyz, src/Programs.f90:38-85). */
int gemsgpu_set_positions(gemsgpu_ctx* ctx, int sys, const double* pos);
/* Replace velocities / accelerations only. */
int gemsgpu_set_velocities(gemsgpu_ctx* ctx, int sys, const double* vel);
int gemsgpu_set_accelerations(gemsgpu_ctx* ctx, int sys, const double* acel);
/* Copy state back; any pointer may be NULL.  epot_atoms is per atom (n). */
int gemsgpu_download(gemsgpu_ctx* ctx, int sys, double* pos, double* vel,
                     double* force, double* epot_atoms);
int gemsgpu_download_acel(gemsgpu_ctx* ctx, int sys, double* acel);

/* box_setvars (src/Program_Types.F90:126-141) + set pbc: boxed=0 removes
 * the box (O(N^2) lists, src/Neighbour.F90:591-606). */
int gemsgpu_set_box(gemsgpu_ctx* ctx, int sys, int boxed, const double L[3],
                    const int pbc[3]);
/* nb_dcut, the Verlet skin (src/Neighbour.F90:237). */
int gemsgpu_set_skin(gemsgpu_ctx* ctx, int sys, double skin);
/* Displacement measure of the skin test.  mic=0 is the reference's
 * test_update (src/Neighbour.F90:1305-1346): raw pos - pos_old, so an atom
 * wrapped into the box by do_pbc triggers a rebuild; mic=1 (default) takes
 * the minimum image and skips those rebuilds (same forces, fewer rebuilds). */
int gemsgpu_set_skin_mode(gemsgpu_ctx* ctx, int sys, int mic);
/* 0 = full list, newton off (OpenMP default); 1 = half list, newton on
 * (the serial default, src/Neighbour.F90:160-171).  gemsgpu_get_list returns
 * the list of the chosen mode in the reference's order.  The force kernels
 * always sum over the full list: with the reaction added to j, a half list
 * gives every atom the same force, density and energy (src/TB.F90:432-441,
 * 542-552; src/Pairs.F90:248-252), up to summation order. */
int gemsgpu_set_list_mode(gemsgpu_ctx* ctx, int sys, int half);
int gemsgpu_set_precision(gemsgpu_ctx* ctx, int sys, int prec);

/* lj_set / plj_set (src/Pairs.F90:198-205, 282-291) for the type pair
 * (ti,tj): epsilon (eV), sigma (A), cut-off (A).  shifted_force=1 selects
 * plj; eshift (eV) is an optional constant energy shift per pair (0 = lj). */
int gemsgpu_set_lj(gemsgpu_ctx* ctx, int sys, int ti, int tj, double eps,
                   double sigma, double rcut, int shifted_force,
                   double eshift);
/* slj_set (src/Pairs.F90:374-401): LJ to rs (A), then a polynomial tail
 * sa4 (r - rc)^4 + sa8 (r - rc)^8 that vanishes with its slope at the
 * derived cut-off rc = rs - 32 u(rs) / (11 u'(rs)).  Pairs of a system may
 * mix lj, plj and slj (slj_interact, Pairs.F90:403-470); FP64 systems. */
int gemsgpu_set_slj(gemsgpu_ctx* ctx, int sys, int ti, int tj, double eps,
                    double sigma, double rs);
/* wca_set (src/Pairs.F90:495-506): Weeks-Chandler-Andersen, LJ cut at
 * 2**(1./6.) sigma (the exponent a single-precision literal, as the
 * reference evaluates it) and shifted up by eps (wca_interact,
 * Pairs.F90:508-589).  Same as gemsgpu_set_lj with that cut-off and
 * eshift = -eps. */
int gemsgpu_set_wca(gemsgpu_ctx* ctx, int sys, int ti, int tj, double eps,
                    double sigma);
/* sm1_set (src/Pairs.F90:916-923): smooth step of depth eps (eV) that rises
 * from -eps at r1 to 0 at r2 (A), the cut-off; the force keeps the factor r
 * of sm1_interact (Pairs.F90:957).  FP64 systems. */
int gemsgpu_set_sm1(gemsgpu_ctx* ctx, int sys, int ti, int tj, double r1,
                    double r2, double eps);
/* `interact g1 feels g2` (src/Interaction.f90:69-76, 128-131): after a pair
 * setter for (ti, tj), the pair acts on the atoms of type ti only (give each
 * group its own type).  Energies count the feeling side's half, as the
 * reference's.  Not with the virial or a piston (no pair virial).  The
 * direction turned off stays off: a later set_lj / set_slj / set_wca /
 * set_sm1 of the same pair changes its parameters on the feeling side only. */
int gemsgpu_set_feels(gemsgpu_ctx* ctx, int sys, int ti, int tj);
/* Pair virial W = sum_i r_i (x) F_i (inq_virial, Inq_Properties.F90:439-527)
 * accumulated by the force kernels of an lj/plj/slj or SMA-TB system (on=1;
 * FP64, or FP32 per pair with FP64 accumulation in mixed precision; SMA-TB
 * forces are central pair forces, and the library sums the complete virial
 * where TB.F90:548-564 omits the i-side term); the pistons switch it on. */
int gemsgpu_set_virial(gemsgpu_ctx* ctx, int sys, int on);
/* smatb_set (src/TB.F90:106-170): A, xi (eV), p, q, r0, rci, rce (A).  The
 * device derives the tail polynomial coefficients. */
int gemsgpu_set_smatb(gemsgpu_ctx* ctx, int sys, int ti, int tj, double A,
                      double xi, double p, double q, double r0, double rci,
                      double rce);
/* Tersoff 1988 parameters (Tersoff.f90:56-59 form): A, B (eV), lambda1,
 * lambda2, beta, n, c, d, h, R, D, chi. */
int gemsgpu_set_tersoff(gemsgpu_ctx* ctx, int sys, const double prm[12]);

/* ------------------------------------------------------------ forces */

/* interact (src/Interaction.f90:135-241): on the first call build the list
 * (update, Neighbour.F90:1242-1299), later run test_update
 * (Neighbour.F90:1305-1346); zero and compute forces and per-atom energies.
 * *epot (may be NULL) receives the system's potential energy (internal
 * units), *rebuilt (may be NULL) whether the list was rebuilt. */
int gemsgpu_forces(gemsgpu_ctx* ctx, int sys, double* epot, int* rebuilt);
/* update: rebuild the neighbour list now. */
int gemsgpu_update(gemsgpu_ctx* ctx, int sys);
/* Export the list: nn[n] and the column-major list (cap x n) like
 * ig%list(i,m) (src/Neighbour.F90:116-117); indices are 0-based atom
 * indices of the system.  *cap_needed gets the largest nn. */
int gemsgpu_get_list(gemsgpu_ctx* ctx, int sys, int* nn, int* list, int cap,
                     int* cap_needed);
/* Number of list rebuilds so far (nupd_vlist, src/Neighbour.F90:246). */
int gemsgpu_get_nupd(gemsgpu_ctx* ctx, int sys, int64_t* nupd);

/* ------------------------------------------------------------ integrators */

int gemsgpu_set_vv(gemsgpu_ctx* ctx, int sys, double dt);
/* `evolve pred_corr_5` (src/Integration.F90:143-145): the fifth-order
 * Nordsieck predictor-corrector, nordsieck_predictor as step a and
 * nordsieck_corrector as step b (Integration.F90:1192-1268), on the scaled
 * derivatives acel..acel4 that the atoms keep (zero for new atoms; read and
 * written by gemsgpu_chp_read / gemsgpu_chp_write). */
int gemsgpu_set_pred_corr(gemsgpu_ctx* ctx, int sys, double dt);
/* set_ermak (src/Integration.F90:909-961): dt (ps), gamma (1/ps), T (K).
 * The device draws its normals from a counter-based Philox4x32-10 stream
 * keyed by seed (production mode). */
int gemsgpu_set_ermak(gemsgpu_ctx* ctx, int sys, double dt, double gamma,
                      double temp, uint64_t seed);
/* `evolve brownian temp gama` (src/Integration.F90:146-149, 834-882):
 * overdamped Langevin steps x += F/m dt/gamma + r sqrt(2 kB T dt/gamma / m),
 * v = (x - x_old)/dt, all in step b.  dt (ps), T (K), gamma (1/ps); normals
 * from the Philox stream keyed by seed, or the parity stream below. */
int gemsgpu_set_brownian(gemsgpu_ctx* ctx, int sys, double dt, double temp,
                         double gamma, uint64_t seed);
/* Thermostats that run after the system's integrator, as a second `evolve`
 * line does (integration_stepb, src/Integration.F90:264-275).  scalvel
 * (set_scalvel :1271-1340): v *= (T0/T)^(0.5/steps) every step, T from the
 * centre-of-mass-free kinetic energy; upto >= 0 selects scalvel_after,
 * which scales only while |T - T0| > upto T0; upto < 0 selects scalvel. */
int gemsgpu_set_scalvel(gemsgpu_ctx* ctx, int sys, double temp, int steps,
                        double upto);
/* andersen (set_andersen / andersen, :1343-1395): each atom collides with
 * probability nu dt (nu in 1/ps; the deck's default is 20) and takes
 * velocities of scale sqrt(kB T / (3N)^2) / sqrt(m), the reference's factor;
 * Philox stream keyed by seed. */
int gemsgpu_set_andersen(gemsgpu_ctx* ctx, int sys, double temp, double nu,
                         uint64_t seed);
int gemsgpu_clear_thermostat(gemsgpu_ctx* ctx, int sys);
/* Parity mode: the next step of an Ermak (step a) or Brownian (step b)
 * system consumes these normals (6 per atom: r1,r2 for x, y, z in atom
 * order, as rang() draws them in ermak_a, Integration.F90:988-993; cbrownian
 * uses each pair's r1) instead of the device stream. */
int gemsgpu_set_ermak_normals(gemsgpu_ctx* ctx, int sys,
                              const double* normals);
/* FIRE (Bitzek 2006) with the per-atom mixing of FIRE.f90:107-114: dt0,
 * dt_max (ps).  Velocities are zeroed. */
int gemsgpu_set_fire(gemsgpu_ctx* ctx, int sys, double dt0, double dtmax);
/* set_lgf (src/Integration.F90:486-525), `evolve piston_lgf xyz*`: constant
 * pressure and temperature Langevin dynamics of Gronbech-Jensen & Farago
 * (J. Chem. Phys. 141, 194108, 2014) with an isotropic piston on the
 * volume.  dt (ps), T (K), target pressure (atm), particle friction pgama0
 * and piston friction pgamav (1/ps), piston mass pmass; lgf_stepa/stepb
 * (:527-650) per step.  The box moves on the device every step (its cell
 * grid re-planned within 15% growth); FP64 lj/plj/slj or SMA-TB systems in
 * a box periodic in x, y and z.  Production noise: Philox4x32-10 keyed by seed. */
int gemsgpu_set_lgf(gemsgpu_ctx* ctx, int sys, double dt, double temp,
                    double press_atm, double pgama0, double pgamav,
                    double pmass, uint64_t seed);
/* set_lkd (src/Integration.F90:329-355), `evolve piston_lkd`: the Langevin
 * piston of Kolb & Dunweg (J. Chem. Phys. 111, 4453, 1999) as lkd_stepa /
 * lkd_stepb (:357-484) state it; arguments and restrictions as
 * gemsgpu_set_lgf. */
int gemsgpu_set_lkd(gemsgpu_ctx* ctx, int sys, double dt, double temp,
                    double press_atm, double pgama0, double pgamav,
                    double pmass, uint64_t seed);
/* One integrator per coordinate (`evolve piston_lgf x|y|z` and
 * `evolve ermak_x|y|z`, Integration.F90:157-186): a G-JF piston on one box
 * length (set_lgf_flex, :652-696; lgf_flex_stepa/b, :698-830; arguments as
 * gemsgpu_set_lgf) or Ermak dynamics of one coordinate (set_ermak with a
 * coordinate, :909-961; ermak_a_x/b_x, :1033-1105).  axis 0, 1, 2 = x, y,
 * z; each call adds one integrator (a system that had another kind of
 * integrator starts an empty set), all with the same dt, at most one per
 * coordinate; a coordinate without one keeps its velocity.  The pistons
 * move their lengths with the volume of the step's start, as the reference
 * updates the volume after all of them.  Pistons need an FP64 lj/plj/slj or
 * SMA-TB system periodic along their axis. */
int gemsgpu_add_lgf_axis(gemsgpu_ctx* ctx, int sys, int axis, double dt,
                         double temp, double press_atm, double pgama0,
                         double pgamav, double pmass, uint64_t seed);
int gemsgpu_add_ermak_axis(gemsgpu_ctx* ctx, int sys, int axis, double dt,
                           double gamma, double temp, uint64_t seed);
/* Parity mode: the next step_a of a piston or per-coordinate system
 * consumes these normal pairs, in the order rang() draws them.  Isotropic
 * piston (lgf_stepa, Integration.F90:561-590): 2 + 6 n values, the
 * piston's pair, then a pair per atom and coordinate (the first value of
 * each pair is used).  Per-coordinate integrators, in the order they were
 * added: a piston's pair then a pair per atom, or an Ermak coordinate's
 * pair per atom.  LKD piston: 6 n + 2 pairs, stepa's pair per atom
 * coordinate and piston pair, then stepb's piston pair and pair per atom
 * coordinate.  NULL returns to the device stream. */
int gemsgpu_set_lgf_normals(gemsgpu_ctx* ctx, int sys, const double* normals);
/* The box lengths (A) as the device holds them (moved by a piston). */
int gemsgpu_get_box(gemsgpu_ctx* ctx, int sys, double L[3]);
/* The pair virial of the last force evaluation (eV, row-major 3x3) and the
 * pressure tensor (sum m v v + W) / V in atm (inq_pressure,
 * Inq_Properties.F90:529-573; write_pressure, Output.F90:767-770). */
int gemsgpu_virial(gemsgpu_ctx* ctx, int sys, double* out9);
int gemsgpu_pressure(gemsgpu_ctx* ctx, int sys, double* out9);

/* integration_stepa / integration_stepb (src/Integration.F90:243-301):
 * the algorithm's half step followed by do_pbc (Set_Properties.f90:444-470). */
int gemsgpu_step_a(gemsgpu_ctx* ctx, int sys);
int gemsgpu_step_b(gemsgpu_ctx* ctx, int sys);
/* dinamic (src/Programs.f90:114-167) without output: nsteps of
 * step_a / interact / step_b on the device, no host round trip per step
 * (CUDA-graph captured).  Requires a prior gemsgpu_forces call or runs one. */
int gemsgpu_md_steps(gemsgpu_ctx* ctx, int sys, int nsteps);

/* Potential energy, kinetic energy with the centre-of-mass velocity removed
 * and temperature (inq_pot_energy, inq_kin_energy, inq_temperature,
 * src/Inq_Properties.F90:358-437).  Energies in eV, T in K. */
int gemsgpu_energy(gemsgpu_ctx* ctx, int sys, double* epot_ev,
                   double* ekin_ev, double* temp);
/* max |F| over the system's atoms, eV/A. */
int gemsgpu_fmax(gemsgpu_ctx* ctx, int sys, double* fmax_ev);

/* ------------------------------------------------------------ batches */

/* Advance nsys systems together: every kernel of a step covers all of them
 * in one launch (uneven sizes packed by a block map). */
int gemsgpu_batch_md_steps(gemsgpu_ctx* ctx, const int* sys, int nsys,
                           int nsteps);
/* FIRE-relax nsys systems together to max|F| < fmax (eV/A) or maxit
 * iterations; iters[k] (may be NULL) receives each system's count. */
int gemsgpu_batch_fire(gemsgpu_ctx* ctx, const int* sys, int nsys,
                       double fmax, int maxit, int* iters);
/* Energies of nsys systems (arrays of nsys; any may be NULL). */
int gemsgpu_batch_energy(gemsgpu_ctx* ctx, const int* sys, int nsys,
                         double* epot_ev, double* ekin_ev, double* temp);
/* Positions and/or velocities of nsys systems in one call (the state
 * hand-off of group_switch_vectorial, src/Groups.F90:553-585, for a whole
 * batch): pos[k] / vel[k] are interleaved xyz host arrays of system k (the
 * pointer arrays or any entry may be NULL).  All copies are queued together
 * and the call synchronises once; with page-locked host arrays the copies
 * run at the link's DMA speed.  Setting positions makes the next force
 * call test the skin, as gemsgpu_set_positions does. */
int gemsgpu_batch_set_state(gemsgpu_ctx* ctx, const int* sys, int nsys,
                            const double* const* pos, const double* const* vel);
/* The reverse, plus the energies of gemsgpu_batch_energy (any output may be
 * NULL). */
int gemsgpu_batch_get_state(gemsgpu_ctx* ctx, const int* sys, int nsys,
                            double* const* pos, double* const* vel,
                            double* epot_ev, double* ekin_ev, double* temp);

/* ------------------------------------------------------------ minimisation */

/* L-BFGS minimisation in place (lbfgs_minimizator + lbfgs,
 * src/Quasi_Newton.f90:77-160, 349-663): Liu-Nocedal limited-memory BFGS
 * with m correction pairs (1..8; the reference uses 5) and the More-Thuente
 * line search of mcsrch/mcstep (ftol 1e-4, gtol 0.9, 100 evaluations per
 * search); f is E_pot in eV, g = -F in eV/A (get_fg).  Stops when
 * |g| / int(max(1, |x|)) <= eps (the reference: 1e-8), after itermax
 * iterations, or when a line search fails (xtol: relative interval width,
 * 1e-15 in the reference).  The systems end at their last evaluated point
 * with its forces.  Per system (arrays of nsys, any may be NULL): iters =
 * iterations, nfun = function evaluations, status = 0 converged, 1
 * iteration limit, -1 line search failed; emin_ev = final E_pot (eV).  The
 * batch form relaxes nsys systems together, each with its own search. */
int gemsgpu_lbfgs(gemsgpu_ctx* ctx, int sys, int m, double eps, double xtol,
                  int itermax, int* iters, int* nfun, int* status, double* emin_ev);
int gemsgpu_batch_lbfgs(gemsgpu_ctx* ctx, const int* sys, int nsys, int m,
                        double eps, double xtol, int itermax, int* iters,
                        int* nfun, int* status, double* emin_ev);

/* ------------------------------------------------------------ NEB */

/* Nudged elastic band (neb, neb_linin, nebfce, nebvel: src/NEB.f90:58-355)
 * on nimg image systems sys[0..nimg-1] of the same atoms and force field.
 * The images listed in `fixed` (increasing 0-based indices, two or more)
 * hold their positions; the others are first set on the straight line
 * between the neighbouring fixed ones.  iters iterations of velocity Verlet
 * with unit masses on the NEB force (improved tangent, spring constant k_ev
 * in eV/A^2) with the quick-min velocity projection, time step
 * sqrt(2 * 5e-5 / F_rms) from the initial band; the end images do not move.
 * As in the reference the last image's energy enters the tangent choice as
 * 0 until the end.  On return the systems hold the final band with its
 * forces; dt_out (may be NULL) gets the time step (ps) and eimg_ev (nimg,
 * may be NULL) each image's potential energy (eV). */
int gemsgpu_neb(gemsgpu_ctx* ctx, const int* sys, int nimg, const int* fixed,
                int nfixed, double k_ev, int iters, double* dt_out,
                double* eimg_ev);

/* ------------------------------------------------------------ checkpoints */

/* Per-system checkpoint (write_chp / read_chp, src/Checkpoint.F90:154-244):
 * positions, velocities, accelerations and the Nordsieck derivatives
 * acel2..acel4 in the GEMS layout plus the integrator state (Philox step
 * counter, FIRE dt/alpha/counters, the box
 * and the G-JF piston's force, velocity and last noise) and the
 * rebuild count, in a caller-owned host buffer of gemsgpu_checkpoint_size
 * bytes.  Loading into a system of the same size restores that state; the
 * next interact rebuilds the neighbour list, as the reference's does after
 * read_chp. */
int gemsgpu_checkpoint_size(gemsgpu_ctx* ctx, int sys, size_t* bytes);
int gemsgpu_checkpoint_save(gemsgpu_ctx* ctx, int sys, void* buf, size_t bytes);
int gemsgpu_checkpoint_load(gemsgpu_ctx* ctx, int sys, const void* buf,
                            size_t bytes);

/* GEMS's own checkpoint file (write_chp / read_chp, src/Checkpoint.F90:
 * 154-244): the Fortran unformatted records of the reference, so GEMS and
 * this library resume each other's runs.  The caller supplies (write) or
 * receives (read) what the file holds beyond the system's state: the
 * algorithm index, step counters, the LCG generator state (idum, iy, ix of
 * write_chpseed, src/Random.F90:178-184) and the output counters.
 * gemsgpu_chp_write needs the forces at the current positions (the piston
 * values it writes close the last step as lgf_stepb does); with buf NULL it
 * only reports the size in *written.  gemsgpu_chp_read takes a system of the
 * file's atom count, restores positions, velocities, accelerations, the box
 * and the piston velocities; the next force evaluation rebuilds the list
 * and a piston takes its force from that evaluation's virial, as the
 * reference does after read_chp.  Higher derivatives are written as zero
 * and ignored on reading. */
typedef struct {
  int32_t current, step, nsteps;
  int32_t rng[3];   /* lcg idum, iy, ix */
  double nframe, time, dm_steps, pnframe, ptime;
  int32_t frame;
} gemsgpu_chp_info;
int gemsgpu_chp_write(gemsgpu_ctx* ctx, int sys, const gemsgpu_chp_info* info,
                      void* buf, size_t bytes, size_t* written);
int gemsgpu_chp_read(gemsgpu_ctx* ctx, int sys, const void* buf, size_t bytes,
                     gemsgpu_chp_info* info);

/* ------------------------------------------------------------ pools */

/* A pool runs a changing set of systems (one force-field kind and precision)
 * through one captured CUDA graph: its launch maps have fixed capacity and
 * are rewritten when the set changes, so admitting or retiring a system
 * costs no graph capture.  Capacity: max_systems systems, max_atoms atoms
 * and max_cells cells in total; each run advances chunk_steps MD steps.
 * lanes / variant fix the force kernels' launch shape (see gemsgpu_autotune).
 * Replaces the per-rank dinamic loops of parallel_tempering2 and drives the
 * serving loop; no single reference routine corresponds. */
int gemsgpu_pool_create(gemsgpu_ctx* ctx, int max_systems, int64_t max_atoms,
                        int64_t max_cells, int ff, int prec, int lanes,
                        int variant, int chunk_steps, gemsgpu_pool** out);
int gemsgpu_pool_destroy(gemsgpu_pool* pool);
/* Set the active systems (replaces the previous set); new members get their
 * first list and forces. */
int gemsgpu_pool_set(gemsgpu_pool* pool, const int* sys, int nsys);
/* Advance the active set by nchunks x chunk_steps steps (FIRE systems that
 * have converged stay frozen). */
int gemsgpu_pool_run(gemsgpu_pool* pool, int nchunks);

/* ------------------------------------------------------------ serving */

/* A serving loop over one pool.  Jobs wait in a queue and are admitted, in
 * arrival order but skipping jobs that do not fit, while the running jobs
 * hold at most max_atoms atoms and max_jobs slots (admission by memory
 * footprint).  Every gemsgpu_server_step admits what fits, advances all
 * running jobs by one chunk on the device (their work overlaps in the same
 * kernels), and retires finished jobs: their energy, max|F|, iterations and
 * final positions stay on the host until gemsgpu_server_forget.  Each job's
 * result does not depend on which other jobs share its chunks.  GEMS itself
 * has no serving mode; this sits on the same kernels as gemsgpu_md_steps. */
int gemsgpu_server_create(gemsgpu_ctx* ctx, int max_jobs, int64_t max_atoms,
                          int prec, int lanes, int variant, int chunk_steps,
                          gemsgpu_server** out);
int gemsgpu_server_destroy(gemsgpu_server* srv);
int gemsgpu_server_submit(gemsgpu_server* srv, const gemsgpu_job* job,
                          int64_t* job_id);
int gemsgpu_server_step(gemsgpu_server* srv, int* n_running, int* n_queued,
                        int* n_finished);
/* state: GEMSGPU_JOB_*; results are filled once DONE (pos_out: 3n). */
int gemsgpu_server_poll(gemsgpu_server* srv, int64_t job_id, int* state,
                        double* epot_ev, double* fmax_ev, int* iters,
                        double* pos_out);
int gemsgpu_server_forget(gemsgpu_server* srv, int64_t job_id);

/* ------------------------------------------------------------ replicas */

/* One exchange round of parallel tempering (parallel_tempering2,
 * src/ReplicaExchange.f90:27-150) among nrep Ermak systems.  temps[k] is the
 * k-th temperature (any order the caller keeps fixed) and sys_of_temp[k] the
 * system currently at temps[k].  In round `round` index k pairs with k+par
 * (k even) or k-par (k odd), par = +1 for even rounds and -1 for odd ones;
 * the lower index accepts with min(1, exp(-(b_k - b_k')(U_k' - U_k))).  An
 * accepted swap exchanges the two systems' temperature labels and rescales
 * their velocities by sqrt(T_new/T_old) -- the configurations stay on the
 * device (the reference moves them between MPI ranks).  Uniforms come from
 * Philox(seed, round, k) or, if `uniforms` is not NULL, from uniforms[k].
 * sys_of_temp is updated in place; *accepted gets the number of swaps. */
int gemsgpu_replica_exchange(gemsgpu_ctx* ctx, int nrep, int* sys_of_temp,
                             const double* temps, int round, uint64_t seed,
                             const double* uniforms, int* accepted);

/* The decision of one exchange round alone, in host arithmetic (no device,
 * no context): epot_ev[k] is the potential energy (eV) of the replica at
 * temps[k]; partner[k] receives the temperature index whose replica moves
 * to temps[k] (k itself when no swap).  Same rule and uniforms as
 * gemsgpu_replica_exchange, so every rank of a multi-GPU run that has
 * gathered the same energies reaches the same decisions. */
int gemsgpu_remd_decide(int nrep, const double* epot_ev, const double* temps,
                        int round, uint64_t seed, const double* uniforms,
                        int* partner, int* accepted);
/* Give nsys Ermak systems new temperatures, rescaling each one's velocities
 * by sqrt(T_new/T_old) (the second half of an accepted exchange). */
int gemsgpu_retemper(gemsgpu_ctx* ctx, int nsys, const int* sys,
                     const double* temps);

/* ------------------------------------------------------------ no allocation */

/* Largest system gemsgpu_smatb_forces_noalloc accepts. */
#define GEMSGPU_NOALLOC_MAX_ATOMS 16384

/* SMA-TB forces for callers that cannot allocate device memory -- a host
 * that hands the library only buffers from its own fixed device budget, or
 * code running where cudaMalloc/cudaFree are not allowed (they synchronise
 * the device and are refused during CUDA-graph stream capture).  This entry
 * point has no counterpart in the reference (GEMS has no device code); it
 * computes what smatb_interact computes for one species (A, xi, p, q, r0,
 * rci, rce as in gemsgpu_set_smatb) from caller-owned DEVICE buffers:
 *   d_pos   positions, 3n doubles, GEMS interleaved layout (read);
 *   d_force forces, 3n doubles (written), internal units;
 *   d_epot  per-atom potential energy, n doubles (written), internal units.
 * boxed/L/pbc as in gemsgpu_set_box.  Work is queued on `stream` (a
 * cudaStream_t, NULL = the legacy default stream) and not waited for.
 * It allocates nothing: its only scratch is a fixed file-scope device array
 * of 2 x GEMSGPU_NOALLOC_MAX_ATOMS doubles (256 KiB) that every GPU loading
 * the library holds until exit.  n > GEMSGPU_NOALLOC_MAX_ATOMS returns
 * GEMSGPU_ERR_FULL without launching.  The first call on a device looks up
 * the array's device address, so make that first call before any stream
 * capture.  That address is kept for the life of the process: after
 * cudaDeviceReset (or anything else that destroys the device's primary
 * context) do not call this function on that device again.  All calls share
 * the array: calls that overlap on the GPU (two streams, or two host
 * threads) race; calls ordered on one stream do not. */
int gemsgpu_smatb_forces_noalloc(const double* d_pos, int n, int boxed,
                                 const double L[3], const int pbc[3],
                                 double A, double xi, double p, double q,
                                 double r0, double rci, double rce,
                                 double* d_force, double* d_epot,
                                 void* stream);

/* ------------------------------------------------------------ tuning */

/* Time the system's force kernels over the candidate launch shapes (lanes
 * per atom 1..32; for mixed SMA-TB the variant bits: bit 0 species
 * constants in shared memory (1) or registers (0, single species), bit 1 a
 * register-capped build with more blocks per SM (four per SM), bit 2 with
 * bit 1 a force pass capped at three blocks per SM) and keep the fastest.  reps timed
 * evaluations per candidate.  No reference counterpart (GEMS has no device
 * code); the choice changes summation order only. */
int gemsgpu_autotune(gemsgpu_ctx* ctx, int sys, int reps, int* lanes_out,
                     int* variant_out, double* best_ms);
/* The same search timed on nsys systems launched together (one shape for
 * all of them: the best shape of a batch differs from a lone system's). */
int gemsgpu_batch_autotune(gemsgpu_ctx* ctx, const int* sys, int nsys, int reps,
                           int* lanes_out, int* variant_out, double* best_ms);
/* Set the launch shape by hand (lanes: 1,2,4,...,32; variant 0..3, 6, 7). */
int gemsgpu_set_lanes(gemsgpu_ctx* ctx, int sys, int lanes, int variant);

/* ------------------------------------------------------------ measurement */

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or CUDA events against the library's.  No reference counterpart. */
int gemsgpu_get_stream(gemsgpu_ctx* ctx, void** stream);
/* Kernel launches issued by ctx so far (graph replays count their kernel
 * nodes).  No reference counterpart: GEMS has no device code. */
int gemsgpu_get_launch_count(gemsgpu_ctx* ctx, int64_t* launches);
/* Time the force kernels of `sys` on the context's stream with CUDA events:
 * reps back-to-back evaluations after one warm-up; out_ms[0] = mean time of
 * the first force kernel (density pass for SMA-TB, bond records for
 * Tersoff), out_ms[1] = mean time of the second (force pass; Tersoff's
 * gather; 0 if none), out_ms[2] = mean list rebuild time.
 * Replaces timer_dump's per-step wall time (src/Errors.f90:128-172). */
int gemsgpu_time_kernels(gemsgpu_ctx* ctx, int sys, int reps, double* out_ms);
/* The same for nsys systems launched together (one launch shape). */
int gemsgpu_batch_time_kernels(gemsgpu_ctx* ctx, const int* sys, int nsys,
                               int reps, double* out_ms);

/* Measured issue-rate roofs of the pipes the force kernels use, on one
 * device: out[0] FP32 FMA TFLOP/s, out[1] FP64 FMA TFLOP/s, out[2] MUFU
 * ex2 Gop/s, out[3] MUFU rsqrt Gop/s.  No counterpart in the reference: it
 * gives the compute roofs that the kernels' achieved rates are set against. */
int gemsgpu_measure_peaks(int device, double* out);

#ifdef __cplusplus
}
#endif

#endif /* GEMSGPU_H */
