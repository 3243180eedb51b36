/*
 * simox_gpu.h -- C ABI of the B200 force / charge / integrate path for SIMOX.
 *
 * Drop-in boundary for the per-step subroutines that SIMOX's Fortran main loop
 * (main.f90:29-34 start-up, main.f90:41-61 regular loop, main.f90:63-84
 * oxidation loop) calls by reference.  Every entry point below names the
 * reference subroutine it replaces.  A Fortran ISO_C_BINDING shim with the same
 * subroutine names copies the PTCL array of derived types field-wise into the
 * plain arrays used here (the reference types are not BIND(C)).
 *
 * Conventions
 *  - Every function returns an int status: SIMOX_OK (0) or a negative
 *    SIMOX_E_* code.  simox_status_string() gives the text, and for the codes
 *    that correspond to a reference STOP the text is that STOP message.
 *  - Atom arrays are in the caller's (original) atom order, 0-based.
 *    Vectors (positions, velocities, forces) are interleaved [n][3] doubles,
 *    i.e. q(i)%xx(1:3) of the reference stored contiguously per atom.
 *  - Species ids are the reference's: Al=1, Ni=2, Fe=3, O=4, H=5.
 *  - Units are the reference's: Angstrom, eV, amu, e, time unit 10.1805 fs.
 *  - A context owns device-resident state (positions, velocities, forces,
 *    charges, cell lists, PME grids) and one CUDA stream.  Contexts are not
 *    thread-safe, like the reference's serial code.
 *  - Energies are accumulated in FP64 in both precision modes.
 */
#ifndef SIMOX_GPU_H
#define SIMOX_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- limits and constants (datafmt.f90:20-31) -------------------------- */
#define SIMOX_NATOM   5     /* Al, Ni, Fe, O, H                 datafmt.f90:29 */
#define SIMOX_NMETAL  3     /* Al, Ni, Fe                       datafmt.f90:30 */
#define SIMOX_NRDF    200   /* radial distribution bins         datafmt.f90:31 */
#define SIMOX_NPT_MAX 500   /* reference per-cell atom limit    datafmt.f90:20 */
#define SIMOX_NNB_MAX 500   /* reference per-atom neighbour limit datafmt.f90:22 */
/* RDF histogram: rdf[(id_i-1) + 5*(id_j-1) + 25*bin], bin = INT(r/dr) in
 * [0, SIMOX_NRDF+1]; the Fortran array pair%rdf(5,5,201) is the same memory
 * shifted by one bin (Fortran index k <-> C bin k). */
#define SIMOX_RDF_LEN (SIMOX_NATOM * SIMOX_NATOM * (SIMOX_NRDF + 2))

/* ---- status codes ------------------------------------------------------ */
#define SIMOX_OK                 0
#define SIMOX_E_ARG             -1  /* bad argument / null pointer */
#define SIMOX_E_CUDA            -2  /* CUDA runtime or cuFFT failure */
#define SIMOX_E_NOMEM           -3  /* device allocation failed */
#define SIMOX_E_CELL_OVERFLOW   -4  /* "=== Cell particle limit crashed !!! ===" cellsort.f90:75 */
#define SIMOX_E_NBR_OVERFLOW    -5  /* "=== neighbor particle limit crashed !!! === " ctip.f90:153 / force.f90:79 */
#define SIMOX_E_UNKNOWN_PAIR    -6  /* "=== Unknown particle pair ===" force.f90:73 */
#define SIMOX_E_UNKNOWN_ELEMENT -7  /* "# Unknown element" force.f90:346 */
#define SIMOX_E_BRENT           -8  /* "# **** Brent solver limit breached *** " ctip.f90:302 */
#define SIMOX_E_CELL_TOO_SMALL  -9  /* "==== Error - unitcell is too small ..." main.f90:271 */
#define SIMOX_E_CAPACITY       -10  /* more atoms than the context was created for */
#define SIMOX_E_POSITION       -11  /* a coordinate is not finite or far outside the box */
#define SIMOX_E_CG_LIMIT       -12  /* CG iteration cap reached (cap is opt-in; reference has none) */
#define SIMOX_E_FFT_SIZE       -13  /* PME grid dimension not usable */
#define SIMOX_E_STATE          -14  /* call order violated (e.g. FORCE before CELL_SORT) */
#define SIMOX_E_NO_DEVICE      -15  /* no CUDA device / library built without one */
#define SIMOX_E_UNSUPPORTED    -16  /* hetero-metal pair forms (METAL_HETERO, AL_NI,
                                       eam.f90:38-168) are not on the GPU path */
#define SIMOX_E_SCRATCH_LIMIT  -17  /* simox_cell_sort_noalloc: more than 65,536 cells
                                       or a link stride above 4,096 */
#define SIMOX_E_IO             -18  /* checkpoint file cannot be opened, read or written,
                                       is not a checkpoint, or its box differs */
#define SIMOX_E_RNG            -19  /* VV_NVT2_STOCH: a random-force draw rejected 100
                                       polar-method attempts (probability 3e-67) */
#define SIMOX_E_SYNC           -20  /* a device-wide wait inside a kernel gave up after its
                                       iteration limit (its CTAs did not all arrive) */

/* ---- precision modes --------------------------------------------------- */
#define SIMOX_FP64   0   /* every term in FP64 (the FP64 GPU oracle path) */
#define SIMOX_MIXED  1   /* pair terms and PME grids FP32; sums, energies,
                            CG dots, residuals and projection FP64 */

/* ---- option flags (simox_setup.flags) ----------------------------------- */
#define SIMOX_FLAG_REFERENCE_LIMITS 0x1  /* enforce Nnb_max = 500 like the reference */

/* ---- potential parameters: derived types of datafmt.f90:54-74 ---------- */
typedef struct {            /* TYPE METL  datafmt.f90:65-68 */
    double r_e, f_e, rho_e, rho_s, alpha, beta, A, B, kappa, lambda;
    double Fn[4], Fm[4], Fp[4];
    double eta, Fe;
} simox_metl;

typedef struct {            /* TYPE POTN  datafmt.f90:54-56 */
    double xm, qmin, qmax, chi, J, xi, Z;
    double fafb[SIMOX_NATOM][4];   /* fafb[j-1][k-1] = param(i)%fafb(j,k) */
} simox_potn;

typedef struct {            /* TYPE OXID  datafmt.f90:70-74 */
    double r_e[SIMOX_NATOM], alph[SIMOX_NATOM], beta[SIMOX_NATOM];
    double A[SIMOX_NATOM], B[SIMOX_NATOM], kapp[SIMOX_NATOM], lamb[SIMOX_NATOM];
    double F0[4], F1[4], F2[4], F3[4], F4[4];
    double re[5], rmax[5];
    double fe, gamm, nu;
} simox_oxid;

typedef struct {
    simox_metl eam[SIMOX_NMETAL];
    simox_potn param[SIMOX_NATOM];
    simox_oxid oxygn;
} simox_potential;

/* ---- system set-up: the parts of AMNT/STAT that fix array shapes -------- */
typedef struct {
    int    n_atoms;      /* Nset%Npt_all                                        */
    int    capacity;     /* atoms the context can hold (>= n_atoms; 0 = n_atoms) */
    double box[3];       /* Nset%box (Angstrom); positions live in [-L/2, L/2)  */
    int    fft[3];       /* Nset%fft: PME grid K1 x K2 x K3                     */
    int    pme_order;    /* B-spline order: 4 (reference, cubic), 6 or 8         */
    double rcut;         /* sys%Rcut; Ewald a = 3.8/Rcut (main.f90:254)          */
    int    precision;    /* SIMOX_FP64 or SIMOX_MIXED                            */
    int    npt_max;      /* per-cell capacity (0 = SIMOX_NPT_MAX)                */
    int    nnb_max;      /* per-atom neighbour capacity (0 = 1024)               */
    int    device;       /* CUDA device ordinal                                  */
    int    flags;        /* SIMOX_FLAG_*                                         */
    double skin;         /* Verlet skin (A) of the internal pair list: 0 = 1.0,
                            < 0 = rebuild from the reference cells every call  */
} simox_setup;

/* Energies of TYPE STAT (datafmt.f90:59-63), all FP64, eV. */
typedef struct {
    double Eself, Edir, Erec, Epair, Egroup, Ectip;
    double mv2;          /* sum m v^2 (amu A^2 / time-unit^2 = eV)                 */
} simox_energies;

/* Outcome of one CTIP_SOLVER call. */
typedef struct {
    int    n_cg;         /* nonlinear-CG iterations (ctip.f90:169-190)           */
    int    n_line;       /* line-search (Brent) evaluations summed over iterations */
    double error;        /* final MAXVAL(|p|)*|alpha|                             */
    double q_sum;        /* total charge after the solve                          */
} simox_ctip_report;

/* Options of the device-resident main loop (main.f90:40-84, TAG_SET main.f90:376). */
typedef struct {
    double dt;           /* time step in internal units (fs / 10.180505306645389) */
    int    thermostat;   /* 0 = NVE (VV_NVE2), 1 = Berendsen (VV_NVT2_BEREND)     */
    double T_given;      /* target temperature in eV (K * kB)                     */
    int    freq_new;     /* charges when MOD(step, freq_new) == 1; <= 0: never    */
    int    freq_sort;    /* cell sort when MOD(step, freq_sort) == 0              */
    int    reflect;      /* 1 = VV_NVE1_REFLECT (oxidation mode top wall)         */
    int    charge_every_step; /* 1 = CTIP on every step (driver flag)             */
    int    accumulate_rdf;    /* 1 = accumulate the RDF histogram in FORCE        */
    int    freq_stat;         /* energies (FP64) on steps with MOD(step, freq_stat)
                                 == 0 (TAG_SET's status rule); <= 0: every step  */
    int    thermo_stoch;      /* with thermostat = 1: 1 = the stochastic pair
                                 VV_NVT1_STOCH / VV_NVT2_STOCH (tag%thermo_stoch)
                                 instead of VV_NVE1 / VV_NVT2_BEREND; such steps
                                 run without CUDA graphs                         */
    double alpha;             /* friction of the stochastic thermostat (Nset%alpha) */
    unsigned long long seed;  /* seed of its random forces (see simox_vinit)      */
} simox_md_opts;

/* Oxidation-mode charge events (main.f90:63-84, Nset%N_o2, z_new, q_crit of
 * config.prm lines 19-21): on every charge step REMOVE_RIGID_MOTION,
 * OXIDE_CHECK and, when it is due, NEW_O2 run between CELL_SORT and
 * CTIP_SOLVER.  The reference draws the new dimers from RANDOM_NUMBER; here
 * from the seeded generator of simox_vinit, stream (1 << 63 | step). */
typedef struct {
    int    n_o2;         /* O2 dimers per insertion (Nset%N_o2); 2 n_o2 atoms     */
    double z_new;        /* height of the new dimers' centres (Nset%z_new), A     */
    double q_crit;       /* OXIDE_CHECK charge threshold (Nset%q_crit), e         */
    unsigned long long seed;  /* seed of the dimer positions                      */
} simox_oxidation;

typedef struct simox_ctx simox_ctx;

/* ---- parameter tables --------------------------------------------------- */
/* POTENTIAL_SETUP (datafmt.f90:142-262): fills the hard-coded Al/Ni/Fe/O/H
 * tables and the Slater fafb coefficients.  Host-only; needs no GPU. */
int simox_default_potential(simox_potential* pot);

/* Text of a status code; reference STOP message where one exists. */
const char* simox_status_string(int status);

/* Library / build description string (host-only). */
const char* simox_version(void);

/* ---- context lifetime (READ_INPUT allocation, main.f90:96-260) ---------- */
int simox_create(const simox_setup* setup, const simox_potential* pot, simox_ctx** out);
int simox_destroy(simox_ctx* ctx);

/* Host <-> device state copies.  x, v, f: [n][3]; q: [n]; id: [n].
 * Any pointer may be NULL to skip that field (id is required on the first
 * set_state).  n may differ from the previous call (NEW_O2, datafmt.f90:98)
 * up to the capacity. */
int simox_set_state(simox_ctx* ctx, int n, const int* id, const double* x,
                    const double* v, const double* f, const double* q);
int simox_get_state(simox_ctx* ctx, int n, int* id, double* x, double* v,
                    double* f, double* q);
int simox_get_natoms(simox_ctx* ctx, int* n);

/* ---- cells: cellsort.f90 ------------------------------------------------ */
/* CELL_HIERARCHY (cellsort.f90:3-36): the 13-cell half stencil, 1-based cell
 * ids, pair[(id-1)*13 + n-1] = cell(id)%pair(n).  ncell_out[3] = Nset%Ncell. */
int simox_cell_hierarchy(simox_ctx* ctx, int* ncell_out, int* pair);
/* CELL_SORT (cellsort.f90:53-80): bins atoms on the device; cell membership
 * and in-cell order are bit-exact to the reference. */
int simox_cell_sort(simox_ctx* ctx);
/* Exports the bins in the reference layout: npt[c] = cell(c+1)%Npt and
 * link[c*link_stride + k] = cell(c+1)%link(k+1) (1-based atom ids). */
int simox_get_cells(simox_ctx* ctx, int* npt, int* link, int link_stride);

/* ---- forces and charges: force.f90, ctip.f90 ---------------------------- */
/* PME_SELF (force.f90:467-517): sets a = 3.8/Rcut, the Ewald self energy and
 * the reciprocal kernel psi (psi(0) = 0, tin-foil). */
int simox_pme_self(simox_ctx* ctx, simox_energies* e);
/* Copies the psi table (K1*K2*K3, x fastest) for checking. */
int simox_get_psi(simox_ctx* ctx, double* psi);
/* CTIP_SOLVER (ctip.f90:3-212): nonlinear CG charge equilibration with the
 * reference's Sigma-g ratio, mean projection, Brent line search on [-1,1]
 * and MAXVAL(|alpha p|) < 1e-3 stop.  Matrix-free: the short-range Slater and
 * erfc couplings are recomputed per pair, the long-range part is the PME
 * potential.  Writes the charges and e->Eself.  max_cg <= 0: no cap. */
int simox_ctip_solve(simox_ctx* ctx, int max_cg, simox_energies* e, simox_ctip_report* rep);
/* FORCE (force.f90:3-361): EAM density, embedding, pair, Ewald real-space and
 * CTIP short-range forces; overwrites forces; sets Epair, Edir, Ectip, Egroup.
 * e: NULL to skip the energies.  Energies are always evaluated with FP64 pair
 * terms (in the mixed precision mode a call with e != NULL runs the FP64 pair
 * kernels), forces of a call with e == NULL use the context's precision.
 * rdf: NULL, or a host histogram of SIMOX_RDF_LEN ints that is incremented. */
int simox_force(simox_ctx* ctx, simox_energies* e, int* rdf);
/* PME (force.f90:364-464): reciprocal-space forces added to the forces, the
 * mean PME force removed, Erec set. */
int simox_pme(simox_ctx* ctx, simox_energies* e);
/* Per-atom EAM density and embedding derivative of the last FORCE call
 * (rho, dF/drho) in original atom order, for checking. */
int simox_get_eam(simox_ctx* ctx, double* rho, double* dFdrho);

/* ---- integrator: vverlet.f90 -------------------------------------------- */
int simox_vv_nve1(simox_ctx* ctx, double dt);                      /* vverlet.f90:74-96   */
int simox_vv_nve1_reflect(simox_ctx* ctx, double dt);              /* vverlet.f90:100-129 */
int simox_vv_nve2(simox_ctx* ctx, double dt, double* mv2);         /* vverlet.f90:132-157 */
int simox_vv_nvt2_berend(simox_ctx* ctx, double dt, double T_given, double* mv2); /* vverlet.f90:160-208 */

/* ---- VINIT and the stochastic thermostat --------------------------------
 * The reference draws its random numbers from Fortran's RANDOM_NUMBER after
 * RANDOM_SEED (main.f90:28), a stream no other program reproduces.  Here every
 * draw is a pure function of (seed, stream, counter) -- the SplitMix64 output
 * mix applied twice, 53 bits scaled into [0, 1) -- so a run is reproducible
 * from its seed on any device and the CPU oracle draws the same numbers.
 * Streams: VINIT (1 << 62 | atom), counter = component; the thermostat at step
 * s (s << 32 | atom), counters 2 (256 d + k), 2 (256 d + k) + 1 for attempt k
 * of component d (atom = index in the caller's order). */
/* VINIT (vverlet.f90:2-71): velocities U[-0.5, 0.5) per component, mean
 * removed, scaled per species to T_given (eV); then FORCE + PME at x - dt v
 * (VV_NVE1 with -dt and zero forces) into f, with x and v restored.  Needs
 * PME_SELF and CELL_SORT first, like the reference.  e (may be NULL): the
 * energies of that FORCE + PME; mv2 (may be NULL): VINIT's as-written sum,
 * every atom's v^2 times the last atom's mass (vverlet.f90:64-69). */
int simox_vinit(simox_ctx* ctx, unsigned long long seed, double T_given, double dt, simox_energies* e,
                double* mv2);
int simox_vv_nvt1_stoch(simox_ctx* ctx, double dt, double alpha);   /* vverlet.f90:237-260 */
/* f += fluct * sqrt(2 alpha T_given / dt) (util.f90:84-101, draws of step
 * `step`), then the damped half kick; mv2 = sum m v^2 */
int simox_vv_nvt2_stoch(simox_ctx* ctx, double dt, double alpha, double T_given,
                        unsigned long long seed, unsigned long long step, double* mv2); /* vverlet.f90:263-296 */

/* ---- checkpoint and status output -----------------------------------------
 * The reference restarts from restart.xyz, written by PRINT_SNAPSHOT
 * (util.f90:22-81) with ES13.6 positions and ES11.4 velocities and forces, so
 * a restarted run does not continue the original trajectory.  The checkpoint
 * keeps every bit of the state: a little-endian file of the 8 bytes
 * "SIMOXCK1", int32 version (1), int32 n, int64 step, double box[3], then
 * int32 id[n], double x[n][3], v[n][3], f[n][3], q[n] (original order). */
int simox_checkpoint_write(simox_ctx* ctx, const char* path, long long step);
/* Reads a checkpoint into the context (as simox_set_state with ids); the box
 * must equal the context's, n its capacity or less.  *step (may be NULL)
 * receives the stored step.  SIMOX_E_IO for a missing, short or foreign file. */
int simox_checkpoint_read(simox_ctx* ctx, const char* path, long long* step);
/* PRINT_STAT's line (util.f90:3-19), host only: time (fs) = step TFM dt,
 * T (K) = mv2 / (3 n) / kB, E_total = E_es + E_eam + mv2 / 2, E_es = Eself +
 * Edir + Erec + Ectip, E_eam, Epair, Egroup, in the reference's
 * FORMAT (ES11.4, 1X, F6.1, 5(1X, ES11.4)) ("******" where F6.1 overflows).
 * buf receives the line without newline (len >= 80). */
int simox_format_status(const simox_energies* e, int n_atoms, int step, double dt, char* buf, int len);

/* ---- device-resident main loop (main.f90:40-84) -------------------------
 * Runs steps first_step .. first_step+nsteps-1 of the reference loop on the
 * device: VV1, CELL_SORT, CTIP_SOLVER (TAG_SET rule), FORCE, PME, VV2/NVT.
 * last: energies of the last energy step of the run (may be NULL); mv2 is the
 * final step's.  rdf: as simox_force, accumulated every step. */
int simox_md_run(simox_ctx* ctx, const simox_md_opts* opts, int first_step,
                 int nsteps, simox_energies* last, int* rdf);

/* ---- timing and counters ------------------------------------------------ */
/* CUDA events on the context's stream around a region of calls. */
int simox_timer_begin(simox_ctx* ctx);
int simox_timer_end(simox_ctx* ctx, float* ms);
/* Per-kernel-family event timing (off by default).  After enabling, each
 * instrumented launch is bracketed by events on the context's stream. */
int simox_profile_enable(simox_ctx* ctx, int on);
/* names: '\n'-separated kernel family names written into buf (may be NULL);
 * ms[k], launches[k] filled for k < cap; *count = number of families. */
int simox_profile_read(simox_ctx* ctx, char* buf, int buflen, double* ms,
                       long long* launches, int cap, int* count);
int simox_profile_reset(simox_ctx* ctx);
/* Total kernels this context has launched since creation. */
int simox_launch_count(simox_ctx* ctx, long long* n);
/* Wait for the context's stream. */
int simox_sync(simox_ctx* ctx);
/* Neighbour statistics of the last list build: max and total list length. */
int simox_neighbor_stats(simox_ctx* ctx, int* max_nnb, long long* total_nnb);
/* Skin-list rebuilds (the device decides when an atom moved more than
 * skin/2) since the skin grid was set up. */
int simox_skin_rebuilds(simox_ctx* ctx, long long* n);

/* ---- parameter adjoint ---------------------------------------------------
 * No counterpart in the reference (which has fixed parameters and no
 * derivatives).  The adjoint model is the FORCE + PME + CTIP_SOLVER physics
 * with the three EAM functions of one metal -- the density f(r) it
 * contributes (eam.f90 ftn), its pair phi(r) with itself (METAL_HOMO) and its
 * embedding F(rho) -- as uniform cubic B-splines of SIMOX_SPLINE_N
 * coefficients each; every term involving oxygen keeps the analytic forms.
 * Its energy is E = Epair + Egroup + U(q*), U the functional CTIP_SOLVER
 * minimises (ctip.f90:307-333) and q* its minimiser (the reference's CG, then
 * Newton steps on the fixed active set to FP64 precision).  Its forces are
 * FORCE + PME at q* (as-written formulas).  All of it is FP64.
 * Gradient layout (SIMOX_NGRAD doubles): phi[64], dens[64], emb[64], then for
 * species 1..5: d/dchi, d/dJ, d/dZ, then d/dxi (zeta) of species 1..5.  The
 * xi derivatives take the Slater coefficients fafb as the functions of xi
 * that datafmt.f90:201-220 defines (as simox_set_ctip_xi sets them). */
#define SIMOX_SPLINE_N 64
#define SIMOX_NGRAD (3 * SIMOX_SPLINE_N + 4 * SIMOX_NATOM)
typedef struct {
    int    metal;            /* species id whose EAM functions are splines (1 = Al) */
    double r0, r1;           /* domain (A) of the f and phi splines; pairs beyond r1 add nothing */
    double rho0, rho1;       /* domain of the embedding spline (extrapolated cubically outside) */
    double phi[SIMOX_SPLINE_N], dens[SIMOX_SPLINE_N], emb[SIMOX_SPLINE_N];
} simox_eam_spline;

typedef struct {
    double E, E_eam, U;      /* E = E_eam + U                                   */
    double loss;             /* sum_i |F_i - T_i|^2 (0 without targets)           */
    double residual;         /* ||P grad_q U|| after the charge refinement         */
    double adj_residual;     /* relative residual of the adjoint CG                */
    int    n_cg, n_newton, n_adjoint;
} simox_adjoint_report;

/* Spline mode of the adjoint model (NULL switches it off).  The context then
 * uses the reference cells' exact list (no skin list). */
int simox_set_eam_spline(simox_ctx* ctx, const simox_eam_spline* s);
/* CTIP parameters chi, J, Z of species 1..5 (POTN datafmt.f90:54-56). */
int simox_set_ctip_params(simox_ctx* ctx, int species, double chi, double J, double Z);
/* Slater exponent xi (zeta) of species 1..5 (POTN datafmt.f90:57); recomputes
 * the fafb coefficients of every pair involving it (datafmt.f90:201-220).
 * SIMOX_E_ARG for xi <= 0 or xi equal to another species' xi (the cross
 * coefficients divide by xi_a - xi_b). */
int simox_set_ctip_xi(simox_ctx* ctx, int species, double xi);
/* Warm start of simox_adjoint_eval's charge solve (no counterpart in the
 * reference).  on = 1: the solve skips CTIP_SOLVER's nonlinear CG and refines
 * the charges the context holds by the safeguarded Newton steps on their
 * active set -- for a sequence of nearby parameter sets (finite differences,
 * an optimiser's line search), which then all stay on the branch of the
 * charge minimum the held charges lie on.  on = 0 (the default): CG first. */
int simox_adjoint_warm_start(simox_ctx* ctx, int on);
/* Precision of simox_adjoint_eval's forward pair passes (no counterpart in
 * the reference).  SIMOX_FP64 (the default): every term FP64.  SIMOX_MIXED:
 * the pair terms of the density and force passes in FP32 (separations formed
 * in FP64 and rounded once), summed in FP64; the charge solve, PME, the
 * embedding and the adjoint solve and gradients stay FP64.  The context
 * itself stays an FP64 context. */
int simox_adjoint_forward_precision(simox_ctx* ctx, int precision);
/* Charges q*, energy, forces (original order, [n][3], may be NULL) and the
 * gradients of E (grad_E) and of L = sum |F - T|^2 (grad_L; needs f_target
 * [n][3]) with respect to the parameters; either gradient may be NULL.  The
 * loss gradient runs one adjoint CG (FP64) through the charge solve. */
int simox_adjoint_eval(simox_ctx* ctx, const double* f_target, simox_adjoint_report* rep,
                       double* forces, double* grad_E, double* grad_L);
/* simox_adjoint_eval on m distinct contexts (independent snapshots), run
 * concurrently on `threads` host threads (<= 0: one per context, at most 16),
 * each context on its own stream.  Any of the array arguments may be NULL, as
 * may any entry.  Returns the first non-zero status in context order. */
int simox_adjoint_eval_many(simox_ctx* const* ctxs, int m, const double* const* f_target,
                            simox_adjoint_report* reps, double* const* forces,
                            double* const* grad_E, double* const* grad_L, int threads);

/* ---- launch-shape tuning -------------------------------------------------
 * No counterpart in the reference (a GPU launch choice).  Results do not
 * depend on it: every atom's force is summed by one warp in the same order
 * whatever the CTA split. */
typedef struct {
    int force_splits;    /* CTAs per skin cell in the mixed pair passes, 1..16 (default 1) */
    int half_list;       /* get only: 1 when the current pair order keeps each pair once (mixed
                            precision, skin list, one metal species plus oxygen); the neighbour
                            statistics then count pairs, not list entries of both atoms      */
} simox_tuning;
int simox_set_tuning(simox_ctx* ctx, const simox_tuning* t);
int simox_get_tuning(simox_ctx* ctx, simox_tuning* t);

/* ---- batched independent systems ----------------------------------------
 * No counterpart in the reference (which runs one system per process): many
 * independent systems of different sizes, each a context created and set up
 * by the caller (simox_create, simox_set_state, simox_pme_self,
 * simox_cell_sort, charges), advanced together.  After one eager step per
 * system, one MD step of ALL systems becomes one CUDA graph and every
 * further step is a single graph launch.  In the per-pass mode (the
 * default) the graph launches each kernel of the step ONCE for all systems
 * (a work list of system blocks; each block reads its system's arguments
 * from a device table) and each FFT once per group of systems with the same
 * PME grid (batched cuFFT plans); this needs every system to take the same
 * kernel sequence (mixed precision on the half list, the same PME order,
 * thermostat and reflect setting), and a batch whose systems differ falls
 * back to the per-system mode: one graph branch per system holding its own
 * launches.  The contexts must live on one device, use the same
 * freq_new/freq_sort/freq_stat, and have freq_new = 0 (charges held).  The
 * batch does not own the contexts; destroy it before its members, and after
 * changing a member's atom set destroy and recreate it. */
typedef struct simox_batch simox_batch;
int simox_batch_create(int nsys, simox_ctx* const* ctxs, simox_batch** out);
int simox_batch_destroy(simox_batch* b);
/* Steps first_step .. first_step+nsteps-1 of main.f90:40-61 for every system;
 * opts[k] and last[k] (may be NULL) belong to system k. */
int simox_batch_md_run(simox_batch* b, const simox_md_opts* opts, int first_step, int nsteps,
                       simox_energies* last);
/* Autotuner: times `trial_steps` batch steps (real MD steps, after one
 * untimed step) for each candidate rule "force_splits = clamp(ceil(target /
 * skin cells), 1, 16)" with target in {0 (one CTA per cell), 148, 296, 592,
 * 1184} CTAs, keeps the fastest and applies it to every system.  times_ms[5]
 * (may be NULL) receives the per-step time of each candidate; *best the index. */
int simox_batch_autotune(simox_batch* b, const simox_md_opts* opts, int first_step, int trial_steps,
                         double* times_ms, int* best);
/* Kernels launched by the batch (graph kernel nodes counted per replay; a
 * cuFFT execution counts as one). */
int simox_batch_launch_count(simox_batch* b, long long* n);
enum { SIMOX_BATCH_PER_PASS = 0, SIMOX_BATCH_PER_SYSTEM = 1 };
/* Request a mode (SIMOX_BATCH_PER_PASS, the default, or
 * SIMOX_BATCH_PER_SYSTEM); takes effect at the next step. */
int simox_batch_set_mode(simox_batch* b, int mode);
/* The mode of the last step the batch launched as a graph. */
int simox_batch_get_mode(simox_batch* b, int* mode);

/* ---- oxidation mode (main.f90:63-84), device-resident ------------------
 * The atom arrays hold the context's capacity, so NEW_O2 appends in place
 * (the reference reallocates, ADD_PTCL datafmt.f90:84-95); an insertion
 * beyond the capacity returns SIMOX_E_CAPACITY.  The only host transfer of a
 * charge event is OXIDE_CHECK's flag. */
/* REMOVE_RIGID_MOTION vverlet.f90:211-234: v -= mean v, z -= mean z (unit
 * masses); FP64 block sums in a fixed order. */
int simox_remove_rigid_motion(simox_ctx* ctx);
/* OXIDE_CHECK util.f90:152-188: *due = 1 when the highest Al atom lies above
 * the highest O atom among the last 2 n_o2 atoms (heights floored at 0) or the
 * largest charge of those O atoms is below q_crit (floored at -10). */
int simox_oxide_check(simox_ctx* ctx, int n_o2, double q_crit, int* due);
/* NEW_O2 datafmt.f90:98-139 with RANDOM_POSITION_O2 util.f90:104-148:
 * appends n_o2 O2 dimers (2 n_o2 atoms of species 4) with centres at height
 * z_new at least sqrt(Lx Ly / n_o2)/2 apart in (x, y), bond 2 A, the y offset
 * as written (equal to the x offset, util.f90:138), v = (0, 0,
 * -sqrt(3 T_given / 16)), f = 0, q = 0.  Draws: stream (1 << 63 | event).
 * SIMOX_E_ARG for "=== Too many new oxygens ===" or no room after 100,000
 * tries; SIMOX_E_CAPACITY beyond the context's capacity.  The new atom set
 * needs simox_cell_sort before FORCE (the reference keeps the new atoms out
 * of its cell lists until its next CELL_SORT). */
int simox_new_o2(simox_ctx* ctx, int n_o2, double z_new, double T_given, unsigned long long seed,
                 unsigned long long event);
/* The oxidation-mode loop main.f90:63-84 (opts->reflect = 1 for
 * VV_NVE1_REFLECT): on each charge step (TAG_SET's freq_new rule, or every
 * step with charge_every_step) REMOVE_RIGID_MOTION, OXIDE_CHECK, NEW_O2 when
 * due (event = step), a CELL_SORT of the moved and new atoms, CTIP_SOLVER;
 * then FORCE, PME and VV_NVE2 / VV_NVT2_BEREND.  *n_inserted (may be NULL)
 * receives the atoms added; simox_get_natoms gives the new count. */
int simox_md_run_oxidation(simox_ctx* ctx, const simox_md_opts* opts, const simox_oxidation* ox,
                           int first_step, int nsteps, simox_energies* last, int* rdf, int* n_inserted);

/* ---- allocation-free cell binning ---------------------------------------
 * No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory -- programs whose GPU memory belongs to another
 * allocator (a framework's caching pool, or an arena reserved at start-up),
 * or per-step loops where cudaMalloc/cudaFree would synchronise the device.
 * Bins n atoms exactly as simox_cell_sort does (same cell membership and
 * in-cell order) without a context and without allocating: the only scratch
 * is a fixed device array of 65,536 cell counters inside the library, which
 * each GPU that loads the library keeps until the process exits.
 *   x_dev       device pointer, positions [n][3] FP64 (centred box coords)
 *   box, rcut   host values; Ncell = INT(box/rcut) as in READ_INPUT
 *   npt_dev     device pointer, Ncell1*Ncell2*Ncell3 ints: atoms per cell
 *   link_dev    device pointer, Ncell*link_stride ints: 1-based atom ids,
 *               ascending within each cell (cell(c)%link layout)
 *   link_stride per-cell row length, 1..4,096 (500 in the reference)
 *   stream      cudaStream_t as void* (NULL: the legacy default stream)
 * Returns SIMOX_E_SCRATCH_LIMIT beyond 65,536 cells or a stride above 4,096,
 * SIMOX_E_CELL_OVERFLOW when a cell holds more than link_stride atoms, and
 * SIMOX_E_CELL_TOO_SMALL for the cell grids simox_create rejects (fewer than
 * 2 cells on an axis, or fewer than 3 on every axis).
 * The call synchronises the stream.  The first call on a device looks up the
 * scratch array's device address with that device current; make that first
 * call before any stream capture.  All calls share the one scratch array, so
 * calls whose work overlaps on the GPU (other threads, other streams) race:
 * serialise them. */
int simox_cell_sort_noalloc(const double* x_dev, int n, const double* box, double rcut,
                            int* npt_dev, int* link_dev, int link_stride, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SIMOX_GPU_H */
