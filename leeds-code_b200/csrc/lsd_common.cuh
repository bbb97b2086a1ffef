// lsd_common.cuh -- shared declarations of the B200 dynamo-step library.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/lsd_b200.h"
#include "lsd_control.cuh"

#define LSD_MAX_KL 8

// complex FP64 stored as double2 (x = re, y = im)
typedef double2 cplx;

#define CUDA_TRY(expr)                                                               \
  do {                                                                               \
    cudaError_t e__ = (expr);                                                        \
    if (e__ != cudaSuccess) {                                                        \
      return lsd_fail(ctx, LSD_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)); \
    }                                                                                \
  } while (0)

// slots of the pinned mirror h_red: corrector sums of squares [0, 8), the tensor-core error
// flag (as int) at 16, tim_cfl_dt at 24, dt staged for the operator build at 32
enum { LSD_HRED_OZERR = 16, LSD_HRED_CFL = 24, LSD_HRED_DT = 32 };

// Kernel families counted for lsd_kernel_launches
#define LSD_LAUNCH(ctx) ((ctx)->launches++)

// operator families (one banded LU + one band Y per l)
enum OpFamily {
  OP_VTOR = 0,  // velocity toroidal  (XTor/YTor, velocity.F90:72-103)
  OP_VPOL = 1,  // velocity poloidal  (XPol/YPol, velocity.F90:104-131)
  OP_VGRE = 2,  // Green's operator   (XGre, velocity.F90:134-146)
  OP_COD = 3,   // codensity          (XC/YC, codensity.F90:37-79)
  OP_COMP = 4,  // composition        (composition.F90:31-54)
  OP_MTOR = 5,  // magnetic toroidal  (magnetic.F90:72-103)
  OP_MPOL = 6,  // magnetic poloidal  (magnetic.F90:104-133)
  OP_NFAM = 7
};

// rotation state on the device (d_rot): the rate, the rate at the last evaluation (the
// inner core's -omega d/dphi), the torques saved by rot_predictor / rot_corrector, the
// torques of the last evaluation, their surface sums (k_products), and dt
enum RotSlot { ROT_OMEGA = 0, ROT_OMEGA_EVAL, ROT_SV_VEL, ROT_SV_MAG, ROT_VEL, ROT_MAG, ROT_SUM_VEL, ROT_SUM_MAG,
               ROT_DT, ROT_NSLOT };

// reference-state bands (d_laps): meshs.F90:364-406
enum LapBand { LAP_COMP = 0, LAP_GRE = 1, LAP_MAGTOR = 2, LAP_MAGPOL = 3, LAP_NBAND = 4 };
// reference-state columns (d_ref, [7][N]): io.F90:559-608
enum RefCol { REF_RHO = 0, REF_XI = 1, REF_DXI = 2, REF_T = 3, REF_DT = 4, REF_ETA = 5, REF_DETA = 6 };

// synthesis group kinds (one CTA group = one output triple)
enum SynthKind {
  SK_VECTOR = 0,  // (q,s,t) -> (r,th,ph)                 tra_qst2rtp  :719-818
  SK_SCALAR = 1,  // a -> a(th,ph)                         tra_spec2phys :472-520
  SK_GRAD3 = 2,   // (dC, C) -> (P dC, P_ C/r, sin1mP iC/r) cod_transform+tra_grad
  SK_GRAD2 = 3,   // C -> (P_ C/r, sin1mP iC/r)            tra_grad :955-1000
};
enum AnalKind {
  AK_VECTOR = 0,  // (r,th,ph) -> (q,s,t)                 tra_rtp2qst :825-949
  AK_SCALAR = 1,  // a -> a                                tra_phys2spec :527-602
};

// theta-Fourier rows: [n][h/2][m-counter c][p = E/O][h%2] per field (complex); a field
// holds N * HB * NM * 4 values.  Half-row pairs keep the rows one FFT block needs together.
__host__ __device__ __forceinline__ size_t four_off(int n, int c, int p, int h, int NM, int HB) {
  return ((((size_t)n * HB + (h >> 1)) * NM + c) * 2 + p) * 2 + (h & 1);
}
// theta-Fourier rows on their way to the analysis (written by the products and r2c
// kernels): [m-counter c][n][h][p = E/O] per field, so one (c, n) row is contiguous along h
// (the analysis contraction runs over h) and a writer of one half-row h fills whole
// 32-byte (E, O) pairs.  Same field size as four_off's.
__host__ __device__ __forceinline__ size_t four_off_a(int n, int c, int p, int h, int N, int Th2) {
  return (((size_t)c * N + n) * Th2 + h) * 2 + p;
}

struct SynthGroup {
  int kind;
  const cplx* in[3];   // spectral inputs [n][H]
  cplx* out[3];        // theta-Fourier outputs [n][NM][Th]
};
struct AnalGroup {
  int kind;
  const cplx* in[3];   // theta-Fourier inputs [n][NM][Th]
  cplx* out[3];        // spectral outputs [n][H]
};

struct lsd_ctx {
  lsd_config cfg;
  int L, M, Mp, N, KL, H, Th, Th2, Ph, Ma, Hc, Hr, NM, P2;
  int HB = 0;                // theta-Fourier half-row pairs, ceil(Th2 / 2)
  int dev = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;
  long long launches = 0;
  std::string err;
  bool owns_stream = false;
  // staged uploads (lsd_stage_coll / lsd_commit_staged): a copy stream, two sets of staging
  // buffers [set][field slot][2 (re, im)][N H] doubles, the fields staged in each set, and
  // events ordering copies, commits and re-use
  cudaStream_t copy_stream = nullptr;
  double* d_stage = nullptr;
  unsigned stage_mask[2] = {0u, 0u};
  int stage_set = 0;
  cudaEvent_t ev_staged[2] = {nullptr, nullptr}, ev_committed[2] = {nullptr, nullptr};

  // host layout
  std::vector<int> hl, hm, hs, thm, mcount, mstart, mlen;
  // device layout
  int *d_l = nullptr, *d_m = nullptr, *d_s = nullptr, *d_mc = nullptr;
  int *d_mstart = nullptr, *d_mlen = nullptr, *d_thm = nullptr, *d_lm2nh = nullptr, *d_bin2c = nullptr;
  int *d_aperm = nullptr;  // [Hc][Hr] analysis thread order
  int *d_sblk_l = nullptr, *d_sblk_nh = nullptr;  // solve blocks: degree, [16] harmonics
  int nsblk = 0;
  int nh_l1m0 = -1, nh_l1m1 = -1;  // toroidal modes of vel_angmomclr
  // device Legendre tables, each [H][Th2] (== Fortran (Th2, H))
  double *d_leg = nullptr;  // 8 tables contiguous, LSD_LEG_* order
  double *d_gp = nullptr, *d_gw = nullptr, *d_sn = nullptr, *d_sn1 = nullptr;
  // FFT twiddles
  double2 *d_tw2 = nullptr;  // e^{+2 pi i k / P2}, k < P2
  double2 *d_twh = nullptr;  // e^{+2 pi i k / Ph}, k < Ph
  int fftG = 1, fftE = 1;     // phi FFT: P2 = fftE * fftG (lanes x registers)
  // radial mesh
  double *d_r = nullptr;       // [7][N]: r^p, p = -3..3
  const double* d_rinv = nullptr;  // 1/r used by the gradient syntheses (d_r + 2N; ones for tra_dth)
  double *d_ones = nullptr;        // [N] ones
  double *d_dr = nullptr;      // [KL][N][2KL+1] bands (column-major per band, like Fortran)
  double *d_r1dr = nullptr;    // [N][2KL+1]
  double *d_radlap = nullptr;  // [N][2KL+1]
  double *d_intr2dr = nullptr; // [N]
  // reference state [7][N] (RefCol order), its bands [LAP_NBAND][N][2KL+1], compr1dr
  // [N][2KL+1] and the weighted integration weights [4][N] (comp, compS, magdiss, veldiss)
  double *d_ref = nullptr, *d_laps = nullptr, *d_compr1dr = nullptr, *d_wts = nullptr;
  bool have_refstate = false;
  // conducting inner core (Nic > 1): its mesh (the same tables as the outer core's on
  // Nic points: r powers [7][Nic], dr bands, radLap, r1dr, intr2dr, weighted weights,
  // reference columns [7][Nic] with eta = 1, reference bands, compr1dr); its field
  // [2][Nic][H] (mag_icTor, mag_icPol) and saved nonlinear terms; the Y bands of its two
  // families [2][Nic][2KL+1][L].  NL = N + Nic - 1 rows per operator (the field families'
  // coupled systems; N rows used by the others).
  int Nic = 1, NL = 0;
  double *d_icr = nullptr, *d_icdr = nullptr, *d_icradlap = nullptr, *d_icr1dr = nullptr, *d_icintr2dr = nullptr;
  double *d_icwts = nullptr, *d_icref = nullptr, *d_iclaps = nullptr, *d_iccompr1dr = nullptr, *d_icyt = nullptr;
  cplx *d_icstate = nullptr, *d_icsv = nullptr;
  // inner-core rotation (rotation.F90), ROT_* slots; Gauss weight x P_0^0 / 2 per theta
  double *d_rot = nullptr, *d_gwP0 = nullptr;
  double rot_inertia = 0.0;
  // operators: LAPACK band LU [fam][L][N][3KL+1] + ipiv [fam][L][N]; Y bands
  // [fam][L][N][2KL+1]; (d_lus / d_ipivs: [fam][N][3KL+1][L] copies, l fastest)
  double *d_lu = nullptr, *d_lus = nullptr, *d_y = nullptr, *d_yt = nullptr;
  int *d_ipiv = nullptr, *d_ipivs = nullptr, *d_info = nullptr;
  double *d_gre = nullptr;   // [L][2][N]
  double *d_gret = nullptr;  // [N][2][L]
  double *d_invg = nullptr;  // [L][4]
  double2 *d_grescr = nullptr;  // [N][L] scratch of k_greens
  bool have_ops = false;
  double op_dt = 0.0;
  // state, nonlinear terms, saved nonlinear terms: [field][N][H] complex
  cplx *d_state = nullptr, *d_nl = nullptr, *d_sv = nullptr;
  // spectral scratch: qst etc. [slot][N][H]
  cplx *d_spec = nullptr;
  int nspec = 0;
  // theta-Fourier scratch: [slot][N][NM][Th]
  cplx *d_four = nullptr;
  int nfour = 0;
  // physical scratch for host-buffer transforms: [slot][N][Ph][Th]
  double *d_phys = nullptr;
  int nphys = 0;
  // host staging (pinned)
  double *h_pin = nullptr;
  size_t h_pin_bytes = 0;
  // reductions
  double *d_red = nullptr;   // small reduction area
  double *d_cpart = nullptr; // corrector: per-warp sums of squares [8][ceil(H / 32)]
  double *h_red = nullptr;   // pinned mirror (64 doubles; slots below)
  // time
  double t = 0.0, dt = 0.0, dterr = 0.0, corr_dt = 0.0, lasterr = 1e99, cfl_dt = 0.0;
  double* d_cfl = nullptr;  // variable dt: [2N] per-shell CFL maxima + tim_cfl_dt
  int it = 0, step = 0;
  bool have_eval = false;
  int tim_pcn = -1;
  // the one-graph step (lsd_step): the device control block and its pinned mirror, the
  // operator build's failure flag, the graph, the streams its conditional bodies are
  // captured on, and the kernels of each section (for lsd_stats.kernel_launches)
  PcDev* d_pc = nullptr;
  PcDev* h_pc = nullptr;
  int* d_opfail = nullptr;
  cudaGraphExec_t g_step = nullptr;
  cudaStream_t cap_stream[2] = {nullptr, nullptr};
  // per stream that launches an evaluation (the context's stream, or a graph-capture
  // stream): two branch streams and the fork / join events of the spectral preparation's
  // independent chains (a stream that joined one capture stays in it until it ends)
  struct Aux { cudaStream_t origin; cudaStream_t s[2]; cudaEvent_t fork, join[2]; };
  std::vector<Aux> eval_aux;
  long long k_begin = 0, k_loop = 0, k_rebuild = 0, k_corr = 0;
  void* oz = nullptr;  // tensor-core path state (lsd_ozaki.cu)
  // tunables besides fftE / fftG and the GEMM tiles (lsd_tune.cu)
  int solve_threads = 128;
  lsd_tuning tuning{};
};

int lsd_fail(lsd_ctx* ctx, int code, const std::string& msg);

// ---- tables (lsd_tables.cu) ----
int lsd_build_tables(lsd_ctx* ctx);
int lsd_build_radial(lsd_ctx* ctx);
int lsd_build_operators(lsd_ctx* ctx);
int lsd_launch_operator_build(lsd_ctx* ctx, const double* dtp, int* status);
// ---- transforms (lsd_sht.cu, lsd_fft.cu) ----
int lsd_launch_synth(lsd_ctx* ctx, const SynthGroup* groups, int ngroups);
int lsd_launch_anal(lsd_ctx* ctx, const AnalGroup* groups, int ngroups);
int lsd_launch_c2r(lsd_ctx* ctx, const cplx* four, double* phys, int nfields);
int lsd_launch_r2c(lsd_ctx* ctx, const double* phys, cplx* four, int nfields);
bool lsd_fft_plan(lsd_ctx* c);
int lsd_launch_products(lsd_ctx* ctx, const cplx* four_in, cplx* four_out);
size_t lsd_products_smem(const lsd_ctx* ctx);
int lsd_launch_qv(lsd_ctx* ctx, const cplx* th, const cplx* ph, cplx* qv1, cplx* qv2);
int lsd_launch_cfl_finish(lsd_ctx* ctx);
// ---- spectral algebra and solves (lsd_solve.cu) ----
int lsd_eval(lsd_ctx* ctx);            // one nonlinear evaluation (device)
int lsd_eval_marked(lsd_ctx* ctx, cudaEvent_t* marks);
int lsd_pred(lsd_ctx* ctx);            // predictor solves (device)
int lsd_corr(lsd_ctx* ctx);            // corrector solves + dterr (device)
int lsd_energy_device(lsd_ctx* ctx, double* out);
int lsd_energy_static(lsd_ctx* ctx, double* out);
int lsd_coll_to_state_n(lsd_ctx* ctx, int rows, const double* re, const double* im, cplx* out);
int lsd_launch_greens(lsd_ctx* ctx, int* d_fail);
int lsd_state_to_coll_n(lsd_ctx* ctx, int rows, const cplx* in, double* re, double* im);
int lsd_diagnostics_device(lsd_ctx* ctx, double* scalars, double* spectra, double* profiles);
int lsd_coll_to_state(lsd_ctx* ctx, const double* re, const double* im, cplx* out);
int lsd_state_to_coll(lsd_ctx* ctx, const cplx* in, double* re, double* im);
int lsd_factor_batch(lsd_ctx* ctx, int n, int kl, int nmat, double* d_ab, int* d_ipiv, int* d_info);
int lsd_operator_solve(lsd_ctx* ctx, int nfield, const int* fields, double* d_data);
int lsd_solve_batch(lsd_ctx* ctx, int n, int kl, int nmat, const double* d_ab, const int* d_ipiv,
                    int nrhs, const int* d_map, double* d_b);

int lsd_umma_selftest(lsd_ctx* ctx, double* maxerr);
// ---- tensor-core (Ozaki) Legendre path (lsd_ozaki.cu) ----
int lsd_ozaki_setup(lsd_ctx* ctx);
void lsd_ozaki_free(lsd_ctx* ctx);
int lsd_ozaki_check(lsd_ctx* ctx);
int* lsd_ozaki_err_flag(lsd_ctx* ctx);
int lsd_ozaki_launch_synth(lsd_ctx* ctx, const SynthGroup* groups, int ngroups);
int lsd_ozaki_launch_anal(lsd_ctx* ctx, const AnalGroup* groups, int ngroups);
bool lsd_ozaki_tiles_ok(int S, int nst, int ctas);
int lsd_ozaki_default_stages(int S);
void lsd_ozaki_default_tiles(int S, int* nst, int* ctas);
void lsd_ozaki_get_tiles(const lsd_ctx* ctx, int* nst, int* ctas);
int lsd_ozaki_set_tiles(lsd_ctx* ctx, int nst, int ctas);
// ---- autotuner (lsd_tune.cu) ----
bool lsd_fft_compiled(int E, int G);
size_t lsd_products_smem_for(int nfields, int P2, int E, int G, int NM);
int lsd_autotune(lsd_ctx* ctx);

// small helpers
static inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
