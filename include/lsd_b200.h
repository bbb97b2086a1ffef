/*
 * lsd_b200.h -- C ABI of the B200-native Leeds Spherical Dynamo timestep hot path.
 *
 * The reference (Leeds-Spherical-Dynamo/leeds-code v3.6.0, Fortran 90) has no runtime
 * plugin API: its seam is the module interface of `transform`, `nonlinear`, `timestep`
 * and the field modules, selected at build time by `TRANSFORM = fftw3`
 * (Scripts/Makefile_template:9,194-196) or `#define _SHTNS`
 * (Scripts/parallel.h_template:17).  Every entry point below replaces one module
 * procedure (cited per function) and is callable from Fortran through ISO_C_BINDING:
 * plain pointers, plain sizes, int status, no C++ or torch types.
 *
 * Array layouts at this boundary are the reference's own Fortran (column-major) ones:
 *   coll  Re(i_N, 0:i_H1)            re[(n-1) + N*nh]            (variables.F90:76-81)
 *   spec  Re(0:i_H1, i_N)            re[nh + H*(n-1)]            (variables.F90:65-70)
 *   phys  Re(i_Th, 0:i_Ph-1, i_N)    p[(j-1) + Th*(i + Ph*(n-1))] (variables.F90:84-86)
 * with the harmonic index nh in the reference's folded order (parallel.h_template:54-80).
 *
 * Status codes: 0 = success; >0 = error class (LSD_E*); lsd_last_error() gives text.
 * No entry point aborts, traps or exits; the reference's `stop 'msg'` becomes a status.
 * A context is single-threaded: one host thread and one CUDA stream per context.
 */
#ifndef LSD_B200_H
#define LSD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define LSD_OK            0
#define LSD_EARG          1   /* bad argument or parameter combination (par_precompute) */
#define LSD_ECUDA         2   /* CUDA runtime error, or no CUDA device                   */
#define LSD_ESINGULAR     3   /* zero pivot in a banded factorisation (mes_lu_find)      */
#define LSD_ENOTCONVERGED 4   /* corrector loop gave up (tim_check_cgce)                 */
#define LSD_ENONFINITE    5   /* NaN/Inf detected in the state                           */
#define LSD_ESTATE        6   /* call out of order (e.g. corrector before predictor)     */
#define LSD_ENOMEM        7   /* device allocation failed                                */

/* ---- fields (coll variables held by the context) ---------------------------------- */
#define LSD_VEL_TOR   0   /* vel_Tor  (velocity.F90)    */
#define LSD_VEL_POL   1   /* vel_Pol                    */
#define LSD_COD_C     2   /* cod_C    (codensity.F90)   */
#define LSD_MAG_TOR   3   /* mag_Tor  (magnetic.F90)    */
#define LSD_MAG_POL   4   /* mag_Pol                    */
#define LSD_COMP_C    5   /* comp_C   (composition.F90) */
#define LSD_NFIELD    6
/* the conducting inner core's field (Nic > 1), coll layout (Nic, H): lsd_set_coll /
 * lsd_get_coll only (magnetic.F90:14-21, io.F90:436-447) */
#define LSD_MAG_IC_TOR 6  /* mag_icTor */
#define LSD_MAG_IC_POL 7  /* mag_icPol */

/* nonlinear terms (outputs of nonlinear.F90), readable with lsd_get_nonlinear */
#define LSD_N_VEL_TOR 0   /* vel_NTor  nonlinear.F90:188 */
#define LSD_N_VEL_POL 1   /* vel_NPol  nonlinear.F90:190 */
#define LSD_N_COD     2   /* cod_NC    nonlinear.F90:276-288 */
#define LSD_N_MAG_TOR 3   /* mag_NTor  nonlinear.F90:443 */
#define LSD_N_MAG_POL 4   /* mag_NPol  nonlinear.F90:441 */
#define LSD_N_COMP    5   /* comp_NC   nonlinear.F90:339-356 */

/* Legendre tables readable with lsd_legendre_table (legendre.F90:41-56), (Th2, H) each */
#define LSD_LEG_P          0
#define LSD_LEG_P_         1
#define LSD_LEG_SIN1MP     2
#define LSD_LEG_LLP_       3
#define LSD_LEG_LLSIN1MP   4
#define LSD_LEG_GWP        5
#define LSD_LEG_GWLLP_     6
#define LSD_LEG_GWLLSIN1MP 7

/* precision of the Legendre contraction */
#define LSD_PREC_FP64   0   /* plain FP64 on the CUDA cores                              */
#define LSD_PREC_OZAKI  1   /* FP64 emulated by int8 slices on tcgen05 tensor cores      */

/* energy diagnostics written by lsd_energies (io.F90:1739-2024 column order) */
#define LSD_E_TIME     0   /* tim_t                                                      */
#define LSD_E_KE       1   /* vel_energy.dat col 2: kinetic energy                       */
#define LSD_E_KE_TOR   2   /* col 3: total toroidal                                      */
#define LSD_E_KE_SYM   3   /* col 4: E_eq_sym                                            */
#define LSD_E_KE_L1    4   /* col 5: E_l=1 (m=0, l even part; variables.F90:837-901)     */
#define LSD_E_KE_TM0   5   /* col 6: E_tor_m=0                                           */
#define LSD_E_KE_DIS   6   /* col 7: viscous dissipation                                 */
#define LSD_E_KE_AX    7   /* col 8: axisymmetric KE                                     */
#define LSD_E_ME       8   /* mag_energy.dat col 2: magnetic energy                      */
#define LSD_E_ME_TOR   9   /* col 3                                                      */
#define LSD_E_ME_SYM  10   /* col 4                                                      */
#define LSD_E_ME_L1   11   /* col 5                                                      */
#define LSD_E_ME_TM0  12   /* col 6                                                      */
#define LSD_E_ME_DIS  13   /* col 7: ohmic dissipation                                   */
#define LSD_E_DIP     14   /* col 8: axial dipole g10                                    */
#define LSD_E_QUAD    15   /* col 9: axial quadrupole g20                                */
#define LSD_E_ME_AX   16   /* col 10: axisymmetric ME                                    */
#define LSD_E_TOPFLX  17   /* top heat flux (io.F90:1773-1783)                           */
#define LSD_E_BOTFLX  18   /* bottom heat flux (io.F90:1785-1794)                        */
#define LSD_NENERGY   19

/* scalars written by lsd_diagnostics (the other time series of io_write2files) */
#define LSD_D_TIME       0   /* tim_t                                                      */
#define LSD_D_VPART      1   /* vel_partition.dat (io.F90:1906-1914): Et, Ep, Etas, Epas,  */
                             /*   Etes, Epes, Etesas, Epesas, sum l E(l), lpol (10 values) */
#define LSD_D_MPART     11   /* mag_partition.dat (io.F90:2018-2020): Et .. Epesas (8)     */
#define LSD_D_CMB       19   /* mag_cmb.dat (io.F90:2036-2145): EPol, ESym, El1, theta,    */
                             /*   phi of the north magnetic pole, Epas, El12 (7)           */
#define LSD_D_NUSC      26   /* codensity Nusselt (io.F90:2158-2243): Nu, T_ro, T_ri,      */
                             /*   dC/dr(ri), dC/dr(ro), Nu_top, Nu_bot, Nu_flux (8)        */
#define LSD_D_NUSX      34   /* the same for composition (8)                               */
#define LSD_D_DYN       42   /* dyn_outputs (io.F90:2355-2399): Rm, Re, Pe, Pe_comp,       */
                             /*   Rossby, M_ratio, Elsasser, Lehnert, fdip, fohm,          */
                             /*   theta_dip, Nusselt, Sherwood (13)                        */
#define LSD_D_DT        55   /* timestep.dat (io.F90:2341-2347): tim_dt, tim_corr_dt,      */
                             /*   tim_cfl_dt (3)                                           */
#define LSD_D_ROT       58   /* rot_torque.dat (io.F90:2249-2266): rot_omega, viscous and   */
                             /*   magnetic torque on the inner core (3)                    */
#define LSD_D_MIC       61   /* mag_ic.dat (io.F90:1933-2024 on mag_icTor/icPol): E, Et,   */
                             /*   Esym, El1, ETm0, EDis, Dip, Quad, Eaxtot (9; Nic > 1)    */
#define LSD_D_MICPART   70   /* its mag_partition.dat line: Et .. Epesas (8; Nic > 1)      */
#define LSD_NDIAG       78
/* spectra (io_save_spectrum / _anelastic / io_save_spectrum1, io.F90:2405-2624), doubles:
 *   velocity: [l = 0..L-1][E, Epol, Etor], then [m = 0..M-1][E, Epol, Etor]
 *   field:    the same;  codensity: [l][E], [m][E];  composition: the same;
 * i.e. 8 (L + M) doubles.  Anelastic velocity: the density-weighted norms
 * (var_coll_normlm_comp) of the compressible q, s, t.
 * profiles (io_rad_profile / io_save_profile, io.F90:2632-2738), [11][N]: r; velocity
 * E, Epol, Etor; field E, Epol, Etor; C, dC/dr (l = 0); Comp, dComp/dr. */

/* ---- configuration: the compile-time `parameters` module as a runtime struct --------- */
typedef struct lsd_config {
  /* resolution (parameters.F90_template:19-23,250) */
  int L, M, Mp, N, Nic, KL;
  /* boundary conditions and switches (parameters.F90_template:45-190) */
  int vel_bc, cod_bc, comp_bc, time_step_control;
  int boussinesq, vel_tstep, cod_tstep, comp_tstep, mag_tstep;
  int precision;            /* LSD_PREC_* for the Legendre contraction                */
  int device;               /* CUDA device ordinal                                    */
  int ozaki_slices;         /* int8 slices per operand for LSD_PREC_OZAKI, 2..8 (0 = 7):
                               S balanced base-256 digits carry 8S - 2 bits (rounded); 5
                               keep 1000-step energies within ~1e-11 of FP64, 7 match FP64 */
  /* physics (parameters.F90_template:29-44) */
  double rratio, alpha, Ra, Ra_comp, Pr, Sc, Pm, E, Hyp;
  /* time integration (parameters.F90_template:229-243) */
  double implicit, timestep, dterr, courant, corr_upper, corr_lower;
  /* sources and fluxes (parameters.F90_template:134-171) */
  double source, source_comp, qi, qo, qi_comp, qo_comp;
  /* inner-core rotation (parameters.F90_template:100-102, rotation.F90) */
  int rot_tstep;            /* b_rot_tstep: step rot_omega with the torques           */
  int rot_force_0;          /* b_rot_force_0: hold rot_omega at zero                  */
  /* no counterpart in the reference (its analogue is FFTW's plan search,
   * transform.fftw3.F90:76-93): 1 = lsd_create times the candidate phi-FFT radices, the
   * tensor-core GEMM's ring depth and CTAs per SM, and the banded solves' threads per CTA
   * on this configuration and keeps the fastest (lsd_get_tuning); 0 = the defaults */
  int autotune;
  int reserved[5];
} lsd_config;

/* derived sizes (parameters.F90_template:251-262; parallel.h_template:54-62) */
typedef struct lsd_sizes {
  int H, Th, Th2, Ph, Ma, Hc, Hr, N, L, M, Mp, KL;
} lsd_sizes;

/* per-call statistics of lsd_step */
typedef struct lsd_stats {
  int steps_done;           /* completed timesteps                                      */
  int correctors;           /* corrector iterations taken in total                      */
  int evaluations;          /* nonlinear evaluations (transforms + products)            */
  int kernel_launches;      /* device kernels launched by this call                     */
  double last_dterr;        /* tim_dterr of the last corrector                          */
  double t, dt;             /* tim_t, tim_dt after the call                             */
} lsd_stats;

/* The loop-control variables of timestep.F90 (tim_t, tim_dt, tim_dterr, tim_corr_dt, the
 * saved lasterr of tim_check_cgce, tim_cfl_dt, tim_it, tim_step, tim_pcn). */
typedef struct lsd_pc_state {
  double t, dt, dterr, corr_dt, lasterr, cfl_dt;
  int it, step, pcn, reserved;
} lsd_pc_state;

typedef struct lsd_ctx lsd_ctx;

/* The tunable launch parameters of a context (lsd_get_tuning / lsd_set_tuning).  No
 * counterpart in the reference (FFTW chooses its own plans there). */
typedef struct lsd_tuning {
  int tuned;             /* 1 when lsd_create timed the candidates (cfg.autotune)          */
  int fft_E, fft_G;      /* phi FFT of P2 = 3M/2 complex points: E-point column DFTs, then
                            G-point row DFTs (both in registers, shared memory between)     */
  int gemm_stages;       /* tensor-core contraction: bulk-copy ring stages (2..4)           */
  int gemm_ctas_per_sm;  /* tensor-core contraction: persistent CTAs per SM (1 or 2)        */
  int solve_threads;     /* banded-solve kernels: threads per CTA (32, 64 or 128)            */
  int reserved[2];
  double ms_fft, ms_gemm, ms_solve;  /* timed ms of the chosen candidates (0: not tuned):
                            one evaluation, one evaluation, one predictor solve             */
} lsd_tuning;

/* The candidates the autotuner times for a configuration (no device work). */
#define LSD_TUNE_MAX 8
typedef struct lsd_tune_space {
  int nfft, fft_E[LSD_TUNE_MAX], fft_G[LSD_TUNE_MAX];
  int ngemm, gemm_stages[LSD_TUNE_MAX], gemm_ctas[LSD_TUNE_MAX];
  int nsolve, solve_threads[LSD_TUNE_MAX];
} lsd_tune_space;

/* Fill cfg with the template parameter values of Scripts/parameters.F90_template. */
int lsd_config_default(lsd_config* cfg);

/* Create a context on cfg->device: radial mesh and FD weights (meshs.F90:116-419),
 * Gauss points (auxiliary/gauwts.f), Schmidt P_l^m tables (legendre.F90:63-128,
 * auxiliary/schnla.f), harmonic layout (variables.F90:103-194) and, at cfg->timestep,
 * the banded operators and their LU factors (velocity/codensity/magnetic *_matrices),
 * all computed in FP64 on the device.  Replaces `initialise` (main.F90:220-380) up to
 * the state load.  Checks par_precompute (parameters.F90_template:274-288). */
int lsd_create(const lsd_config* cfg, lsd_ctx** out);
/* Anelastic reference state: the seven columns of planet_model.txt.in as read by
 * io_load_radial_txtfiles (io.F90:559-608), prof[7][N] = rho, xi = rho'/rho, dxi/dr,
 * T, dT/dr, eta, deta/dr.  Rebuilds the radial bands and weights (mes_rdom_init,
 * meshs.F90:228-415) and the operators.  Only for cfg.boussinesq = 0 contexts; until it
 * is called such a context uses rho = T = eta = 1 with zero gradients. */
int lsd_set_reference_state(lsd_ctx* ctx, const double* prof);
int lsd_destroy(lsd_ctx* ctx);
/* The text of the context's last error; with ctx = NULL, why the calling thread's last
 * lsd_create failed (the configuration rule it broke, or the device it did not find). */
const char* lsd_last_error(const lsd_ctx* ctx);
int lsd_get_sizes(const lsd_ctx* ctx, lsd_sizes* out);

/* Layout and table queries (for bit-identical layout checks).
 * lsd_harmonics: var_H%l, var_H%m, var_H%s (variables.F90:124-152), H ints each.
 * lsd_theta_map: var_Th%m (variables.F90:159-194), 2*Hc ints.
 * lsd_radial_grid: mes_oc%r(:,1) (meshs.F90:135-143), N doubles.
 * lsd_radial_weights: mes_oc%intr2dr (meshs.F90:311-336), N doubles.
 * lsd_gauss: leg_gp, leg_gw (legendre.F90:73), Th doubles each.
 * lsd_legendre_table: one of the LSD_LEG_* tables, (Th2, H) column-major. */
int lsd_harmonics(const lsd_ctx* ctx, int* l, int* m, int* s);
int lsd_theta_map(const lsd_ctx* ctx, int* thm);
int lsd_radial_grid(const lsd_ctx* ctx, double* r);
int lsd_radial_weights(const lsd_ctx* ctx, double* intr2dr);
int lsd_gauss(const lsd_ctx* ctx, double* gp, double* gw);
int lsd_legendre_table(const lsd_ctx* ctx, int which, double* out);

/* ---- state ---------------------------------------------------------------------- */
/* Copy a coll field (Fortran layout) to / from the device.  Replaces the state load
 * (io_load_state, io.F90:349-483) and the refresh before output (io_write2files). */
int lsd_set_coll(lsd_ctx* ctx, int field, const double* re, const double* im);
int lsd_get_coll(lsd_ctx* ctx, int field, double* re, double* im);
/* Streamed inputs (no counterpart in the reference, whose state is host memory): the next
 * state can cross PCIe while the device steps.  lsd_stage_coll enqueues the host-to-device
 * copy of one field (coll layout, as lsd_set_coll) into a staging buffer on the context's
 * copy stream and returns without waiting (pinned host memory makes the copy asynchronous;
 * the host buffer must stay unchanged until a call that waits for the context's work --
 * lsd_step, lsd_energies, lsd_get_coll -- has returned after the commit);
 * lsd_commit_staged makes every field staged since the previous commit the state, on the
 * compute stream after their copies.  Two staging sets alternate, so fields for the next
 * commit can be staged while the step after a commit runs. */
int lsd_stage_coll(lsd_ctx* ctx, int field, const double* re, const double* im);
int lsd_commit_staged(lsd_ctx* ctx);
/* Nonlinear term of the last evaluation (LSD_N_*), coll layout. */
int lsd_get_nonlinear(lsd_ctx* ctx, int which, double* re, double* im);
/* tim_t, tim_dt; setting dt rebuilds the operators (vel/cod/mag_matrices). */
int lsd_set_time(lsd_ctx* ctx, double t, double dt);
int lsd_get_time(const lsd_ctx* ctx, double* t, double* dt, int* step);
/* With cfg.timestep < 0 (d_timestep < 0) lsd_step sets dt itself each step:
 * non_maxtstep (nonlinear.F90:546-615) + tim_new_tstep (timestep.F90:837-870), the
 * operators rebuilt on a change (main.F90:126-134).  out[3] = tim_dt, tim_corr_dt,
 * tim_cfl_dt (io_write_timestep, io.F90:2343-2346). */
int lsd_get_dt_control(const lsd_ctx* ctx, double* out);
/* Inner-core rotation rate rot_omega (the state file's 'omega', io.F90:432) and, read
 * back, out[3] = rot_omega, rot_velTorq, rot_magTorq of the last evaluation
 * (non_rotation, nonlinear.F90:479-538; rotation.F90). */
int lsd_set_rotation(lsd_ctx* ctx, double omega);
int lsd_get_rotation(const lsd_ctx* ctx, double* out);

/* ---- transforms on host buffers (unit parity with transform.fftw3.F90) --------------
 * Each works on all N shells of the context. */
/* tra_spec2phys (transform.fftw3.F90:472-520) */
int lsd_tra_spec2phys(lsd_ctx* ctx, const double* s_re, const double* s_im, double* p);
/* tra_phys2spec (transform.fftw3.F90:527-583, 586-602) */
int lsd_tra_phys2spec(lsd_ctx* ctx, const double* p, double* s_re, double* s_im);
/* tra_qst2rtp (transform.fftw3.F90:719-818) */
int lsd_tra_qst2rtp(lsd_ctx* ctx,
                    const double* q_re, const double* q_im,
                    const double* s_re, const double* s_im,
                    const double* t_re, const double* t_im,
                    double* r, double* th, double* ph);
/* tra_rtp2qst (transform.fftw3.F90:825-949) */
int lsd_tra_rtp2qst(lsd_ctx* ctx, const double* r, const double* th, const double* ph,
                    double* q_re, double* q_im, double* s_re, double* s_im,
                    double* t_re, double* t_im);
/* tra_grad (transform.fftw3.F90:955-1000) */
int lsd_tra_grad(lsd_ctx* ctx, const double* s_re, const double* s_im, double* th, double* ph);
/* tra_dth (transform.fftw3.F90:1006-1031) */
int lsd_tra_dth(lsd_ctx* ctx, const double* s_re, const double* s_im, double* p);
/* tra_qst2rtp_vel (transform.fftw3.F90:611-714), the anelastic velocity: from (q,s,t) and
 * their radial derivatives (qr,sr,tr) the eight fields r, th, ph, dur, qv1, dutr, dupr, qv2 */
int lsd_tra_qst2rtp_vel(lsd_ctx* ctx,
                        const double* q_re, const double* q_im,
                        const double* s_re, const double* s_im,
                        const double* t_re, const double* t_im,
                        const double* qr_re, const double* qr_im,
                        const double* sr_re, const double* sr_im,
                        const double* tr_re, const double* tr_im,
                        double* r, double* th, double* ph, double* dur, double* qv1,
                        double* dutr, double* dupr, double* qv2);

/* ---- device-resident batched transforms (inputs already in HBM) ----------------------
 * d_spec: nbatch spectral fields, interleaved complex, [batch][N][H] (harmonic fastest).
 * d_phys: nbatch physical fields, [batch][N][Ph][Th] (the Fortran phys layout per field).
 * Asynchronous on the context stream. */
int lsd_sht_synth_device(lsd_ctx* ctx, int nbatch, const double* d_spec, double* d_phys);
int lsd_sht_analys_device(lsd_ctx* ctx, int nbatch, const double* d_phys, double* d_spec);

/* ---- time stepping ----------------------------------------------------------------- */
/* vel_matrices + cod_matrices + comp_matrices + mag_matrices at the current dt
 * (velocity.F90:56-168, codensity.F90:37-79, magnetic.F90:62-133). */
int lsd_matrices(lsd_ctx* ctx);
/* One nonlinear evaluation from the current state: *_transform + non_velocity,
 * non_codensity, non_composition, non_magnetic (main.F90:101-124). */
int lsd_nonlinear(lsd_ctx* ctx);
/* vel/cod/comp/mag _predictor (main.F90:136-146) using the last evaluation. */
int lsd_predictor(lsd_ctx* ctx);
/* vel/cod/comp/mag _corrector (main.F90:148-154); *dterr gets tim_dterr. */
int lsd_corrector(lsd_ctx* ctx, double* dterr);
/* nsteps full timesteps (main loop main.F90:100-164: evaluation, predictor, evaluations
 * and correctors until tim_check_cgce converges).  All nsteps run as one launch of one
 * CUDA graph with no host synchronisation inside: a device-side WHILE loop over the
 * steps holds, per step, the evaluation, (d_timestep < 0: non_maxtstep + tim_new_tstep
 * and, when dt changed, the operator rebuild in an IF node), the predictor, and a
 * device-side WHILE loop of corrector evaluations + solves whose condition
 * tim_check_cgce sets on the device.  A step begun by lsd_predictor / lsd_corrector
 * calls is finished first, on the host. */
int lsd_step(lsd_ctx* ctx, int nsteps, lsd_stats* stats);
/* tim_check_cgce (timestep.F90:744-830) on a caller-held loop state, after a corrector
 * whose norm is s->dterr (i_time_step_control 1 or 2 from cfg): s->it becomes 0 when the
 * step is complete or k + 1 when another corrector follows, s->dterr is reset.  Returns
 * LSD_ENOTCONVERGED where the reference gives up (dt -> 0, more than 10 iterations, or a
 * growing error above the limit).  Host only, no device work: lsd_step runs the same
 * function on the device; this entry serves drivers that keep their own loop. */
int lsd_tim_check_cgce(const lsd_config* cfg, lsd_pc_state* s);
/* tim_new_tstep (timestep.F90:837-870) with the CFL limit s->cfl_dt: s->dt takes the next
 * step's dt and *new_dt (tim_new_dt) is 1 when it changed by more than 3 %. */
int lsd_tim_new_tstep(const lsd_config* cfg, lsd_pc_state* s, int* new_dt);
/* Energy diagnostics (io_write_vel_energy / io_write_mag_energy), LSD_NENERGY doubles. */
int lsd_energies(lsd_ctx* ctx, double* out);
/* lsd_energies without any allocation: no counterpart in the reference.  For host codes
 * that cannot allocate when they write diagnostics (device memory fully committed to the
 * state, or work still queued on the stream that a cudaMalloc/cudaFree would stall).  The
 * norm scratch is a static device array sized for N <= 1024 shells (larger N returns
 * LSD_EARG); every call overwrites all of it (nothing carries over between calls).  It is
 * shared by all contexts of a device, so calls that overlap on the GPU (from two host
 * threads or two streams) race on it.  Each call looks the array up (cudaGetSymbolAddress,
 * no allocation); the first lookup in a process may load the module: make the first call
 * before any stream capture. */
int lsd_energies_static(lsd_ctx* ctx, double* out);
/* The other time series, spectra and profiles of io_write2files (io.F90:290-340):
 * io_write_vel_energy / io_write_mag_energy partitions, io_write_cmb, io_write_nussel,
 * io_write_dyn_outputs, io_write_timestep (scalars, LSD_NDIAG doubles, LSD_D_* order);
 * io_save_spectrum / io_save_spectrum_anelastic / io_save_spectrum1 (spectra,
 * 8 (L + M) doubles, or NULL); io_rad_profile / io_save_profile (profiles, 11 N doubles,
 * or NULL).  Layouts above the configuration struct.  Synchronises the context's stream. */
int lsd_diagnostics(lsd_ctx* ctx, double* scalars, double* spectra, double* profiles);

/* ---- ensembles (independent runs at their own resolutions) ---------------------------
 * The reference runs one configuration per job; an ensemble (e.g. a parameter or
 * resolution sweep) is n of them.  lsd_ensemble_create creates one context per config on
 * one device (all cfgs[i].device equal); members are set up, read and diagnosed through
 * the context API (lsd_ensemble_member); lsd_ensemble_step advances every member by
 * nsteps completed steps of main.F90:100-164 as ONE launch of one CUDA graph, in which
 * every member's device-side step loop (lsd_step's graph) is an independent branch, so
 * the members' kernels run concurrently.  stats: n entries, or NULL.  On an error
 * lsd_ensemble_last_error names the member and its message.
 * lsd_ensemble_last_elapsed_ms: device time (CUDA events on the ensemble's stream) of the
 * last lsd_ensemble_step's graph launch. */
typedef struct lsd_ensemble lsd_ensemble;
int lsd_ensemble_create(int n, const lsd_config* cfgs, lsd_ensemble** out);
int lsd_ensemble_destroy(lsd_ensemble* ens);
int lsd_ensemble_size(const lsd_ensemble* ens);
int lsd_ensemble_member(lsd_ensemble* ens, int i, lsd_ctx** ctx);
int lsd_ensemble_step(lsd_ensemble* ens, int nsteps, lsd_stats* stats);
const char* lsd_ensemble_last_error(const lsd_ensemble* ens);
int lsd_ensemble_last_elapsed_ms(const lsd_ensemble* ens, double* ms);

/* ---- batched banded radial solves (timestep.F90:566-588 over every (l,m)) -----------
 * Factorise nmat banded operators A_k (LAPACK band storage with ldab = 3*kl+1, columns
 * of length n, k = 0..nmat-1, overwritten by their LU factors and pivots like dgbtrf,
 * meshs.F90:447-456) and solve nrhs right-hand sides, rhs r using matrix map[r]
 * (dgbtrs, timestep.F90:578-586).  All device pointers; one launch each.
 * d_ab: [nmat][n][3*kl+1] (column-major per matrix), d_ipiv: [nmat][n],
 * d_b: [n][nrhs] (rhs index fastest), d_info: [nmat]. */
int lsd_banded_factor_device(lsd_ctx* ctx, int n, int kl, int nmat, double* d_ab,
                             int* d_ipiv, int* d_info);
int lsd_banded_solve_device(lsd_ctx* ctx, int n, int kl, int nmat, const double* d_ab,
                            const int* d_ipiv, int nrhs, const int* d_map, double* d_b);
/* The context's own factorised Crank-Nicolson operators (built by lsd_create /
 * lsd_set_time at the current dt) applied to caller right-hand sides: for each of the
 * nfield (1..8) fields, X_l x = b for every (l, m) column with tim_zerobc first
 * (tim_invX, timestep.F90:566-588): LSD_COD_C / LSD_COMP_C with tim_lumesh_X (every l),
 * LSD_VEL_TOR with tim_lumesh_flayer_X / _vel_X, LSD_MAG_TOR / LSD_MAG_POL with
 * tim_iclumesh_*_X (Nic = 1; l = 0 not solved, as tim_invX skips it), and LSD_VEL_POL
 * with the reference's fourth-order composite (velocity.F90:369-395, 445-465 without
 * the Y multiply: XGre, XPol, then vel_gre_adjust).  d_data: nfield consecutive device
 * fields in the context's layout, [N][H] complex (re, im interleaved), solved in place;
 * one launch for all fields, on the context's stream (not synchronised). */
int lsd_operator_solve_device(lsd_ctx* ctx, int nfield, const int* fields, double* d_data);

/* ---- autotuning (no counterpart in the reference) ------------------------------------
 * lsd_tune_candidates: the candidates for cfg (the default first in each list), filtered by
 * the compiled radices and the shared-memory limits.  lsd_tune_choose: the selection
 * rule -- the fastest of n timed candidates (ms[]), unless it beats candidate dflt by
 * less than 2 % (timing noise), in which case dflt.  lsd_get_tuning / lsd_set_tuning:
 * the context's parameters (set: validated against its tune space; results may change in
 * the last bits with the FFT radices, not with the other parameters). */
int lsd_tune_candidates(const lsd_config* cfg, lsd_tune_space* out);
int lsd_tune_choose(int n, const double* ms, int dflt);
int lsd_get_tuning(const lsd_ctx* ctx, lsd_tuning* out);
int lsd_set_tuning(lsd_ctx* ctx, const lsd_tuning* in);

/* ---- synchronisation and timing ------------------------------------------------------ */
/* The context's CUDA stream (a cudaStream_t), on which every asynchronous entry point
 * queues its work: for callers that order their own device work (or CUDA events) with
 * the library's.  No counterpart in the reference (single-threaded CPU code). */
int lsd_get_stream(const lsd_ctx* ctx, void** stream);
/* Phase timings (CUDA events on the context stream) of one predictor pass and one
 * corrector solve from the current state; the state advances by that step.  ms[]:
 * 0 spectral q,s,t and curls, 1 Legendre synthesis, 2 phi-FFT + products + FFT,
 * 3 Legendre analysis, 4 spectral tail (curls of N, buoyancy), 5 predictor solves,
 * 6 corrector solves.  *nphase >= LSD_NPHASE on input, = LSD_NPHASE on output.
 * Tracing aid; the reference has only its wall-clock get_time (dyn_mpi.F90:80-93). */
#define LSD_NPHASE 7
int lsd_profile_phases(lsd_ctx* ctx, double* ms, int* nphase);

int lsd_synchronize(lsd_ctx* ctx);
/* Device-side elapsed milliseconds of the last lsd_step / transform call, measured with
 * CUDA events on the context stream. */
int lsd_last_elapsed_ms(const lsd_ctx* ctx, double* ms);
/* Device self-tests of the tensor-core path (diagnostics).  which = 0: one tcgen05 int8
 * product D(128x32) = A(128x64) B(32x64)^T checked against the host product;
 * *result = largest absolute difference (0 expected). */
int lsd_selftest(lsd_ctx* ctx, int which, double* result);
/* Number of device kernels this context has launched so far. */
int lsd_kernel_launches(const lsd_ctx* ctx, long long* count);

#ifdef __cplusplus
}
#endif
#endif /* LSD_B200_H */
