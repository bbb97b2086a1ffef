// lsd_solve.cu -- spectral algebra, the nonlinear evaluation pipeline, the fused
// predictor/corrector banded solves, energies and the batched banded LU API.
//
// Spectral fields live in one layout, [n][H] complex (harmonic fastest), for the whole
// step: the reference's coll <-> spec transposes (var_coll2spec / var_spec2coll,
// variables.F90:246-469) and its MPI all-to-alls therefore do not exist on the device.
// Radial operators act along n with stride H, so a warp of consecutive harmonics reads
// and writes coalesced rows.
#include <cmath>

#include "lsd_banded.cuh"
#include <cstdio>

#include "lsd_common.cuh"

namespace {

// spectral scratch slots
enum SpecSlot {
  S_VQ = 0, S_VS, S_VT, S_VCQ, S_VCS, S_VCT,
  S_BQ, S_BS, S_BT, S_BCQ, S_BCS, S_BCT,
  S_DC, S_DCOMP,
  S_VDQ, S_VDS, S_VDT,  // anelastic: dr q, dr s, dr t of the velocity (var_coll_TorPol2qstderiv)
  S_NSPEC_EVAL
};

struct SpecArgs {
  int N, H, KL, L;
  const int* hl;
  const double* r;      // [7][N]
  const double* r1dr;   // band (2KL+1, N)
  const double* dr1;    // band (2KL+1, N)
};

__device__ __forceinline__ double rtll1(int l) { return l == 0 ? 0.0 : sqrt((double)(l * (l + 1))); }
__device__ __forceinline__ double rtll11(int l) { return l == 0 ? 0.0 : 1.0 / sqrt((double)(l * (l + 1))); }
__device__ __forceinline__ double ll1d(int l) { return (double)(l * (l + 1)); }

// out(n) = sum_j band(KL+1+n-j, j) * in(j), j ascending (var_coll_meshmult order)
__device__ __forceinline__ double2 band_apply(const double* band, int KL, int N, const cplx* in, size_t stride, int n) {
  double2 acc = make_double2(0.0, 0.0);
  const int ldm = 2 * KL + 1;
  for (int j = max(1, n - KL); j <= min(n + KL, N); ++j) {
    double a = band[(size_t)(KL + n - j) + (size_t)ldm * (j - 1)];
    double2 x = in[(size_t)(j - 1) * stride];
    acc.x = acc.x + a * x.x;
    acc.y = acc.y + a * x.y;
  }
  return acc;
}

// q,s,t of a (Tor, Pol) pair: var_coll_TorPol2qst_mag (variables.F90:565-605) with
// s1dr = r1dr, the compressible var_coll_TorPol2qst (:511-556) with s1dr = compr1dr
__global__ void k_qst(SpecArgs a, const double* s1dr, const cplx* tor, const cplx* pol, cplx* q, cplx* s, cplx* t) {
  int nh = blockIdx.x * blockDim.x + threadIdx.x;
  int n = blockIdx.y + 1;
  if (nh >= a.H) return;
  int l = a.hl[nh];
  size_t id = (size_t)(n - 1) * a.H + nh;
  double rm1 = a.r[(size_t)2 * a.N + n - 1];
  double f = ll1d(l) * rm1;
  double2 p = pol[id];
  q[id] = make_double2(p.x * f, p.y * f);
  double2 sv = band_apply(s1dr, a.KL, a.N, pol + nh, a.H, n);
  double w = rtll1(l);
  s[id] = make_double2(sv.x * w, sv.y * w);
  double2 tv = tor[id];
  t[id] = make_double2(-tv.x * w, -tv.y * w);
}

// curl of a qst vector in place: var_coll_qstcurl (variables.F90:713-754)
//   ot = (1/r + dr) s - sqrt(l(l+1))/r q ; os = -(1/r + dr) t ; oq = -sqrt(l(l+1))/r t
__global__ void k_curl(SpecArgs a, const cplx* q, const cplx* s, const cplx* t, cplx* oq, cplx* os, cplx* ot) {
  int nh = blockIdx.x * blockDim.x + threadIdx.x;
  int n = blockIdx.y + 1;
  if (nh >= a.H) return;
  int l = a.hl[nh];
  size_t id = (size_t)(n - 1) * a.H + nh;
  double rm1 = a.r[(size_t)2 * a.N + n - 1];
  double w = rtll1(l) * rm1;
  double2 v = band_apply(a.r1dr, a.KL, a.N, s + nh, a.H, n);
  double2 qv = q[id];
  ot[id] = make_double2(v.x - w * qv.x, v.y - w * qv.y);
  double2 u = band_apply(a.r1dr, a.KL, a.N, t + nh, a.H, n);
  os[id] = make_double2(-u.x, -u.y);
  double2 tv = t[id];
  double w2 = -rtll1(l) * rm1;
  oq[id] = make_double2(tv.x * w2, tv.y * w2);
}

// dC = dr(1) . C (cod_transform, codensity.F90:207)
__global__ void k_drC(SpecArgs a, const cplx* c, cplx* dc) {
  int nh = blockIdx.x * blockDim.x + threadIdx.x;
  int n = blockIdx.y + 1;
  if (nh >= a.H) return;
  dc[(size_t)(n - 1) * a.H + nh] = band_apply(a.dr1, a.KL, a.N, c + nh, a.H, n);
}

// vel_angmomclr (velocity.F90:475-574), stress-free walls: remove the rigid rotations
// carried by the toroidal (l, m) = (1, 0) and (1, 1) modes, the angular momentum being the
// radial integral with the weights w (intr2dr; intr2dr_comp for the anelastic equations).
// One CTA; thread 0 forms the three ratios in the reference's summation order.
__global__ void k_angmom(int N, int H, int nh10, int nh11, const double* r, const double* w, int r2_as_product,
                         cplx* tor) {
  __shared__ double om[3];
  const double* r1 = r + (size_t)4 * N;
  const double* r2 = r + (size_t)5 * N;
  if (threadIdx.x == 0) {
    const double W = 8.0 / 3.0 * 3.1415926535897931;
    double f2 = 0.0, a = 0.0, b = 0.0;
    for (int n = 0; n < N; ++n) f2 = f2 + (r2_as_product ? r1[n] * r1[n] : r2[n]) * w[n];
    om[0] = om[1] = om[2] = 0.0;
    if (nh10 >= 0) {
      for (int n = 0; n < N; ++n) a = a + tor[(size_t)n * H + nh10].x * r1[n] * w[n];
      om[0] = (W * a) / (W * f2);
    }
    if (nh11 >= 0) {
      a = 0.0; b = 0.0;
      for (int n = 0; n < N; ++n) {
        a = a + tor[(size_t)n * H + nh11].x * r1[n] * w[n];
        b = b + tor[(size_t)n * H + nh11].y * r1[n] * w[n];
      }
      om[1] = (2.0 * W * a) / (2.0 * W * f2);
      om[2] = (-2.0 * W * b) / (-2.0 * W * f2);
    }
  }
  __syncthreads();
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    if (nh10 >= 0) tor[(size_t)n * H + nh10].x = tor[(size_t)n * H + nh10].x - om[0] * r1[n];
    if (nh11 >= 0) {
      tor[(size_t)n * H + nh11].x = tor[(size_t)n * H + nh11].x - om[1] * r1[n];
      tor[(size_t)n * H + nh11].y = tor[(size_t)n * H + nh11].y - om[2] * r1[n];
    }
  }
}

// Tail of non_velocity / non_magnetic / non_codensity after the analysis:
//   vel: cq += Ra r Pm^2/Pr C (+ comp) ; NTor = qstllcurlr(t) ; NPol = qstllcurlcurlr(q,s)
//   mag: NPol = qstllcurlr(t) ; NTor = qstllcurlcurlr(q,s)
//   cod: NC = analysed scalar, NC(:, nh=0) += source ;  nh = 0 columns zeroed for vel/mag
//   comp (when stepped): the same with source_comp (nonlinear.F90:341-356)
struct TailArgs {
  SpecArgs s;
  const double* dT0;  // anelastic: dTemp0/dr per shell (buoyancy -Ra T0' Pm^2/Pr); null: Ra r
  double Ra, Ra_comp, Pm2, Pr, Sc, source, source_comp;
  const cplx *vq, *vs, *vt, *bq, *bs, *bt, *cod, *comp;  // comp: nullptr when not stepped
  const cplx *C, *Comp;
  cplx *vNTor, *vNPol, *bNTor, *bNPol, *codNC, *compNC;
};

__global__ void k_tail(TailArgs a) {
  int nh = blockIdx.x * blockDim.x + threadIdx.x;
  int n = blockIdx.y + 1;
  const SpecArgs& s = a.s;
  if (nh >= s.H) return;
  int l = s.hl[nh];
  size_t id = (size_t)(n - 1) * s.H + nh;
  double rm1 = s.r[(size_t)2 * s.N + n - 1];
  double r1 = s.r[(size_t)4 * s.N + n - 1];
  double w = rtll11(l);
  if (nh == 0) {  // l = 0 column zeroed (nonlinear.F90:192-197, 463-472)
    a.vNTor[id] = make_double2(0.0, 0.0);
    a.vNPol[id] = make_double2(0.0, 0.0);
    a.bNTor[id] = make_double2(0.0, 0.0);
    a.bNPol[id] = make_double2(0.0, 0.0);
  } else {
    double2 vt = a.vt[id];
    a.vNTor[id] = make_double2(-vt.x * w, -vt.y * w);
    // buoyancy d2 = Ra*r*(Pm**2)/Pr, anelastic -Ra*Temp0'*(Pm**2)/Pr (nonlinear.F90:158-185)
    double2 q = a.vq[id];
    double2 c = a.C[id];
    const double g = a.dT0 ? a.dT0[n - 1] : r1;
    double d2 = a.Ra * g * a.Pm2 / a.Pr;
    if (a.dT0) d2 = -d2;
    q.x = q.x + d2 * c.x;
    q.y = q.y + d2 * c.y;
    double2 cm = a.Comp[id];
    double d2c = a.Ra_comp * g * a.Pm2 / a.Sc;
    if (a.dT0) d2c = -d2c;
    q.x = q.x + d2c * cm.x;
    q.y = q.y + d2c * cm.y;
    double2 rs = band_apply(s.r1dr, s.KL, s.N, a.vs + nh, s.H, n);
    rs.x = rs.x * w; rs.x = q.x * rm1 - rs.x;
    rs.y = rs.y * w; rs.y = q.y * rm1 - rs.y;
    a.vNPol[id] = rs;
    double2 bt = a.bt[id];
    a.bNPol[id] = make_double2(-bt.x * w, -bt.y * w);
    double2 bq = a.bq[id];
    double2 rb = band_apply(s.r1dr, s.KL, s.N, a.bs + nh, s.H, n);
    rb.x = rb.x * w; rb.x = bq.x * rm1 - rb.x;
    rb.y = rb.y * w; rb.y = bq.y * rm1 - rb.y;
    a.bNTor[id] = rb;
  }
  double2 cv = a.cod[id];
  if (nh == 0) cv.x = cv.x + a.source;
  a.codNC[id] = cv;
  if (a.comp) {
    double2 xv = a.comp[id];
    if (nh == 0) xv.x = xv.x + a.source_comp;
    a.compNC[id] = xv;
  }
}

// ---------------------------------------------------------------------------------------
// Column solves.  A thread owns one harmonic nh of one field: its Re and Im columns
// x(n) = X[n * H + nh] (complex), solved with the same factors like the reference's two
// dgbtrs calls (tim_invX, timestep.F90:566-588).  Consecutive threads take consecutive
// harmonics, so every row access of a warp is one contiguous 512-byte segment, and the
// factors are read from copies with the degree l fastest ([fam][n][band][l]), so a
// warp's factor reads are contiguous too.  Columns stream through register windows:
// KL + 1 rows for the forward elimination with row interchanges, 2 KL + 1 for the banded
// back substitution, right-hand-side rows fetched SPF rows ahead; intermediate columns
// go to per-field scratch in global memory.
// ---------------------------------------------------------------------------------------
struct StepArgs {
  int N, H, KL, L;
  const int* hl;
  const int* hm;
  const double* lus;   // [fam][N][3KL+1][L] LAPACK band factors, l fastest
  const int* ipivs;    // [fam][N][L]
  const double* yt;    // [fam][N][2KL+1][L] Y bands, l fastest
  const double* gret;  // [N][2][L] Green's functions
  const double* invg;  // [L][4]
  cplx* state;  // [field][N][H]
  cplx* nl;
  cplx* sv;
  cplx* work;   // scratch: two column sets per field, [2 field + k][N][H]
  double implicit;
  int cod_bc, comp_bc, vel_bc;
  double qi, qo, qi_comp, qo_comp;
  int comp;
  double* red;  // corrector: [8] sums of squares
  double* cpart;  // corrector: the per-warp sums [8][nwarp] that k_cgce_sums adds up
  int nwarp;      // ceil(H / 32)
  int NL;       // rows per operator in lus / ipivs (N + Nic - 1)
  int Nic;      // inner-core points (> 1: conducting, the field families are coupled)
  cplx* icstate;       // [2][Nic][H] mag_icTor, mag_icPol
  cplx* icsv;          // [2][Nic][H] their saved nonlinear terms
  const double* icyt;  // [2][Nic][2KL+1][L] the inner core's Y bands
  const double* rot;   // ROT_* slots: rot_omega and the rate of the last evaluation
  const double* rtor10;  // vel_setbc_Tor's mes_oc%r(1, nh) at nh of (l, m) = (1, 0)
};

// which solve a grid row performs
enum SolveJob { J_VTOR = 0, J_VPOL, J_COD, J_MTOR, J_MPOL, J_COMP, J_NJOB };

constexpr int SOLVE_THREADS = 128;
constexpr int SPF = 8;  // right-hand-side rows fetched ahead, so that their loads overlap

__device__ __forceinline__ int job_field(int job) {
  return job == J_VTOR ? LSD_VEL_TOR : job == J_VPOL ? LSD_VEL_POL : job == J_COD ? LSD_COD_C
       : job == J_MTOR ? LSD_MAG_TOR : job == J_MPOL ? LSD_MAG_POL : LSD_COMP_C;
}
__device__ __forceinline__ int job_family(int job) {
  return job == J_VTOR ? OP_VTOR : job == J_VPOL ? OP_VPOL : job == J_COD ? OP_COD : job == J_COMP ? OP_COMP
       : job == J_MTOR ? OP_MTOR : OP_MPOL;
}

// band factor element (row r 0-based, column c) of this thread's degree: f[(c LD + r) L]
struct Band {
  const double* f;
  const int* piv;
  int L, LD;
  __device__ double at(int r, int c) const { return __ldg(f + ((size_t)c * LD + r) * L); }
  __device__ int pivot(int c) const { return __ldg(piv + (size_t)c * L); }
};

__device__ __forceinline__ double2 axpy2(double2 y, double a, double2 x) {  // y + a x
  return make_double2(y.x + a * x.x, y.y + a * x.y);
}

// dgbtrs forward part (LAPACK order): for c = 0..N-2 swap rows c and piv(c), then
// x(c+i) -= L(c+i, c) x(c), i <= KL.  in(n) supplies right-hand-side rows in increasing
// n (each once); out(c, y) receives the finished rows.  The right-hand-side rows and the
// factors of a batch of SPF rows are loaded before its arithmetic.
template <int KL, class IN, class OUT>
__device__ __forceinline__ void stream_forward(const Band& B, int N, IN&& in, OUT&& out) {
  constexpr int KD = 2 * KL + 1;
  double2 w[KL + 1];
#pragma unroll
  for (int i = 0; i <= KL; ++i) w[i] = i < N ? in(i) : make_double2(0.0, 0.0);
  for (int c0 = 0; c0 < N; c0 += SPF) {
    double2 buf[SPF];  // rows c0 + KL + 1 + u, requested in increasing order
    int pv[SPF];
    double lf[SPF][KL];
#pragma unroll
    for (int u = 0; u < SPF; ++u) {
      const int c = min(c0 + u, N - 1);
      pv[u] = B.pivot(c);
#pragma unroll
      for (int i = 0; i < KL; ++i) lf[u][i] = B.at(KD + i, c);
    }
#pragma unroll
    for (int u = 0; u < SPF; ++u) buf[u] = c0 + KL + 1 + u < N ? in(c0 + KL + 1 + u) : make_double2(0.0, 0.0);
#pragma unroll
    for (int u = 0; u < SPF; ++u) {
      const int c = c0 + u;
      if (c >= N) break;
      if (c < N - 1) {
        const int p = pv[u] - 1 - c;  // 0..KL
#pragma unroll
        for (int i = 1; i <= KL; ++i)
          if (p == i) { const double2 t = w[0]; w[0] = w[i]; w[i] = t; }
        const double2 temp = make_double2(-w[0].x, -w[0].y);
#pragma unroll
        for (int i = 1; i <= KL; ++i)
          if (c + i < N) w[i] = axpy2(w[i], lf[u][i - 1], temp);
      }
      out(c, w[0]);
#pragma unroll
      for (int i = 0; i < KL; ++i) w[i] = w[i + 1];
      w[KL] = buf[u];
    }
  }
}

// dtbsv (upper, non-unit, bandwidth 2KL; LAPACK column order) on the forward result:
// for c = N-1..0: x(c) = y(c) / U(c, c); x(c-t) -= x(c) U(c-t, c), t <= 2KL.
// in(n) supplies y rows in decreasing n; out(c, x) receives x(c) in decreasing c.
constexpr int SPB = 8;  // rows per batch of the back substitution
template <int KL, class IN, class OUT>
__device__ __forceinline__ void stream_backward(const Band& B, int N, IN&& in, OUT&& out) {
  constexpr int K2 = 2 * KL;
  double2 w[K2 + 1];  // w[t] = pending y(c - t)
#pragma unroll
  for (int t = 0; t <= K2; ++t) w[t] = N - 1 - t >= 0 ? in(N - 1 - t) : make_double2(0.0, 0.0);
  for (int c0 = N - 1; c0 >= 0; c0 -= SPB) {
    double2 buf[SPB];  // rows c0 - K2 - 1 - u
    double uf[SPB][K2 + 1];
#pragma unroll
    for (int u = 0; u < SPB; ++u) {
      const int c = max(c0 - u, 0);
#pragma unroll
      for (int t = 0; t <= K2; ++t) uf[u][t] = B.at(K2 - t, c);  // uf[u][0] = U(c, c)
    }
#pragma unroll
    for (int u = 0; u < SPB; ++u) buf[u] = c0 - K2 - 1 - u >= 0 ? in(c0 - K2 - 1 - u) : make_double2(0.0, 0.0);
#pragma unroll
    for (int u = 0; u < SPB; ++u) {
      const int c = c0 - u;
      if (c < 0) break;
      const double d = uf[u][0];
      const double2 xc = make_double2(w[0].x / d, w[0].y / d);
      out(c, xc);
      const double2 mx = make_double2(-xc.x, -xc.y);
#pragma unroll
      for (int t = 1; t <= K2; ++t) w[t] = axpy2(w[t], uf[u][t], mx);
#pragma unroll
      for (int t = 0; t < K2; ++t) w[t] = w[t + 1];
      w[K2] = buf[u];
    }
  }
}

// W(n) := (Y X)(n) + R(n) with the Y band (2KL+1, N) for every row of a column (tim_multY,
// timestep.F90:640-670) as a pass of its own, eight rows per batch: the batch's X rows,
// band values and R rows are all loaded before any of its rows is stored, so their loads
// overlap (a window advanced one row per streamed row would wait for each X row in turn).
// R may be W (in place) or the nonlinear terms.  Only arrays that no thread of the kernel
// writes (the bands, the nonlinear terms) go through the read-only path (__ldg): that path
// lets the compiler move a load past a store to the same address.
constexpr int MY_BATCH = 8;
template <int KL>
__device__ __forceinline__ void multy_rows(const double* y, int L, const double2* X, const double2* R, double2* W,
                                           size_t rst, int N) {
  constexpr int LDM = 2 * KL + 1, WIN = 2 * KL + MY_BATCH;
  double2 win[WIN];  // X rows n0 - KL .. n0 + MY_BATCH - 1 + KL
#pragma unroll
  for (int t = 0; t < 2 * KL; ++t) {
    const int j = t - KL;
    win[t] = (j >= 0 && j < N) ? X[(size_t)j * rst] : make_double2(0.0, 0.0);
  }
  for (int n0 = 0; n0 < N; n0 += MY_BATCH) {
    double2 r[MY_BATCH];
    double yb[MY_BATCH][LDM];
#pragma unroll
    for (int u = 0; u < MY_BATCH; ++u) {
      const int j = n0 + KL + u;
      win[2 * KL + u] = j < N ? X[(size_t)j * rst] : make_double2(0.0, 0.0);
      const int n = n0 + u;
      r[u] = n < N ? R[(size_t)n * rst] : make_double2(0.0, 0.0);
#pragma unroll
      for (int t = 0; t < LDM; ++t) {
        const int jj = n - KL + t;
        yb[u][t] = (n < N && jj >= 0 && jj < N) ? __ldg(y + ((size_t)jj * LDM + (LDM - 1 - t)) * L) : 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < MY_BATCH; ++u) {
      double2 acc = r[u];
#pragma unroll
      for (int t = 0; t < LDM; ++t) acc = axpy2(acc, yb[u][t], win[u + t]);
      if (n0 + u < N) W[(size_t)(n0 + u) * rst] = acc;
    }
#pragma unroll
    for (int t = 0; t < 2 * KL; ++t) win[t] = win[t + MY_BATCH];
  }
}

__device__ __forceinline__ void warp_partial(double v, const StepArgs& a, int slot);

// per-thread view of one field's columns and this degree's operators
struct ColView {
  double2 *X, *S, *W1, *W2;
  const double2* Nn;
  size_t rst;
  Band B1, B2;       // main operator; Green's operator (poloidal velocity)
  const double* y1;  // Y band of the main family
  const double* g;   // Green's functions: element (n, k) at g[(n 2 + k) L]
  double iG[4];
};

template <int KL>
__device__ ColView col_view(const StepArgs& a, int job, int nh, int l) {
  ColView v;
  const int N = a.N, L = a.L, fam = job_family(job), fld = job_field(job);
  constexpr int LD = 3 * KL + 1, LDM = 2 * KL + 1;
  const size_t F = (size_t)N * a.H;
  v.rst = a.H;
  v.X = a.state + fld * F + nh;
  v.Nn = a.nl + fld * F + nh;
  v.S = a.sv + fld * F + nh;
  v.W1 = a.work + (size_t)(2 * fld) * F + nh;
  v.W2 = a.work + (size_t)(2 * fld + 1) * F + nh;
  const int NL = a.NL;
  v.B1.f = a.lus + (size_t)fam * NL * LD * L + l; v.B1.piv = a.ipivs + (size_t)fam * NL * L + l;
  v.B1.L = L; v.B1.LD = LD;
  v.B2.f = a.lus + (size_t)OP_VGRE * NL * LD * L + l; v.B2.piv = a.ipivs + (size_t)OP_VGRE * NL * L + l;
  v.B2.L = L; v.B2.LD = LD;
  v.y1 = a.yt + (size_t)fam * N * LDM * L + l;
  v.g = a.gret + l;
  for (int i = 0; i < 4; ++i) v.iG[i] = job == J_VPOL ? __ldg(a.invg + (size_t)l * 4 + i) : 0.0;
  return v;
}

// vel_gre_adjust (velocity.F90:445-465): coefficients of the two Green's functions
__device__ __forceinline__ void gre_coeffs(const double* iG, double2 x0, double2 xN, double2& ca, double2& cb) {
  ca = make_double2(iG[0] * x0.x + iG[2] * xN.x, iG[0] * x0.y + iG[2] * xN.y);
  cb = make_double2(iG[1] * x0.x + iG[3] * xN.x, iG[1] * x0.y + iG[3] * xN.y);
}

// The saves of the nonlinear terms, apart from the streamed solves: every load of a batch of
// eight rows is issued before its stores, so that a column's loads overlap.  (Inside the
// streamed passes the right-hand-side callbacks only load: a store there would keep the
// compiler from hoisting the next rows' loads above it, one memory round trip per row.)
// save_terms: S := N.  diff_terms: W := c (N - S), S := N (tim_nlincorr).
constexpr int SAVE_BATCH = 8;
__device__ __forceinline__ void save_terms(const double2* Nn, double2* S, size_t rst, int N) {
  for (int n0 = 0; n0 < N; n0 += SAVE_BATCH) {
    double2 x[SAVE_BATCH];
#pragma unroll
    for (int u = 0; u < SAVE_BATCH; ++u)
      if (n0 + u < N) x[u] = __ldg(Nn + (size_t)(n0 + u) * rst);
#pragma unroll
    for (int u = 0; u < SAVE_BATCH; ++u)
      if (n0 + u < N) S[(size_t)(n0 + u) * rst] = x[u];
  }
}
__device__ __forceinline__ void diff_terms(const double2* Nn, double2* S, double2* W, size_t rst, int N, double c) {
  for (int n0 = 0; n0 < N; n0 += SAVE_BATCH) {
    double2 x[SAVE_BATCH], p[SAVE_BATCH];
#pragma unroll
    for (int u = 0; u < SAVE_BATCH; ++u)
      if (n0 + u < N) { x[u] = __ldg(Nn + (size_t)(n0 + u) * rst); p[u] = S[(size_t)(n0 + u) * rst]; }
#pragma unroll
    for (int u = 0; u < SAVE_BATCH; ++u)
      if (n0 + u < N) {
        S[(size_t)(n0 + u) * rst] = x[u];
        W[(size_t)(n0 + u) * rst] = make_double2(c * (x[u].x - p[u].x), c * (x[u].y - p[u].y));
      }
  }
}

// Predictor (velocity.F90:369-395, codensity.F90:224-234, magnetic.F90:370-408).
// grid (ceil(H / SOLVE_THREADS), J_NJOB).
template <int KL>
__global__ void __launch_bounds__(SOLVE_THREADS) k_predictor(StepArgs a) {
  const int job = blockIdx.y;
  if (job == J_COMP && !a.comp) return;
  if ((job == J_MTOR || job == J_MPOL) && a.Nic > 1) return;  // k_mag_ic
  const int nh = blockIdx.x * blockDim.x + threadIdx.x;
  if (nh >= a.H) return;
  const int l = a.hl[nh], N = a.N, L = a.L;
  const bool zero = (job == J_COD || job == J_COMP);
  const ColView v = col_view<KL>(a, job, nh, l);
  const size_t rst = v.rst;
  const double2 z2 = make_double2(0.0, 0.0);
  // boundary rows of the right-hand side (tim_zerobc; cod_setbc / comp_setbc for l = 0)
  double bc0 = 0.0, bcN = 0.0;
  if (zero && nh == 0) {
    const int bc = job == J_COD ? a.cod_bc : a.comp_bc;
    const double qi = job == J_COD ? a.qi : a.qi_comp, qo = job == J_COD ? a.qo : a.qo_comp;
    if (bc == 1 || bc == 2) bc0 = 1.0;
    else if (bc == 3 || bc == 4) bc0 = qi;
    bcN = (bc == 2 || bc == 4) ? qo : 0.0;
  }
  // vel_setbc_Tor (velocity.F90:291-300): the no-slip inner wall turns with the inner core
  if (job == J_VTOR && l == 1 && a.hm[nh] == 0 && a.vel_bc <= 2) bc0 = a.rot[ROT_OMEGA] * a.rtor10[0];
  auto w1 = [&](int c, double2 x) { v.W1[(size_t)c * rst] = x; };
  auto r1 = [&](int n) { return v.W1[(size_t)n * rst]; };
  if (job == J_VPOL) {
    // Pol := NPol ; zerobc ; invX(XGre) ; Pol := YPol vel_Pol + Pol ; zerobc ; invX(XPol) ;
    // vel_gre_adjust (velocity.F90:369-395, 445-465)
    save_terms(v.Nn, v.S, rst, N);
    auto inA = [&](int n) {
      const double2 x = __ldg(v.Nn + (size_t)n * rst);
      return (n == 0 || n == N - 1) ? z2 : x;
    };
    if (l == 0) {
      for (int n = 0; n < N; ++n) v.X[(size_t)n * rst] = inA(n);
      return;
    }
    stream_forward<KL>(v.B2, N, inA, w1);
    stream_backward<KL>(v.B2, N, r1, [&](int c, double2 x) { v.W2[(size_t)c * rst] = x; });
    multy_rows<KL>(v.y1, L, v.X, v.W2, v.W2, rst, N);  // YPol vel_Pol + Pol, in place
    auto inB = [&](int n) { return (n == 0 || n == N - 1) ? z2 : v.W2[(size_t)n * rst]; };
    double2 x0 = z2, xN = z2;
    stream_forward<KL>(v.B1, N, inB, w1);
    stream_backward<KL>(v.B1, N, r1, [&](int c, double2 x) {
      v.W2[(size_t)c * rst] = x;
      if (c == N - 1) xN = x;
      if (c == 0) x0 = x;
    });
    double2 ca, cb;
    gre_coeffs(v.iG, x0, xN, ca, cb);
#pragma unroll 8
    for (int n = 0; n < N; ++n) {
      const double g1 = __ldg(v.g + (size_t)(2 * n) * L), g2 = __ldg(v.g + (size_t)(2 * n + 1) * L);
      const double2 x = v.W2[(size_t)n * rst];
      v.X[(size_t)n * rst] = make_double2(x.x - ca.x * g1 - cb.x * g2, x.y - ca.y * g1 - cb.y * g2);
    }
    return;
  }
  // other fields: X := Y X + N ; zerobc (+ setbc) ; invX
  const bool solve = (l != 0 || zero);
  save_terms(v.Nn, v.S, rst, N);
  if (!solve) {
    for (int n = 0; n < N; ++n)
      v.X[(size_t)n * rst] = n == 0 ? make_double2(bc0, 0.0) : n == N - 1 ? make_double2(bcN, 0.0)
                                                                         : __ldg(v.Nn + (size_t)n * rst);
    return;
  }
  multy_rows<KL>(v.y1, L, v.X, v.Nn, v.W1, rst, N);  // Y X + N into W1 (solved in place)
  auto inC = [&](int n) {
    if (n == 0) return make_double2(bc0, 0.0);
    if (n == N - 1) return make_double2(bcN, 0.0);
    return v.W1[(size_t)n * rst];
  };
  stream_forward<KL>(v.B1, N, inC, w1);
  stream_backward<KL>(v.B1, N, r1, [&](int c, double2 x) { v.X[(size_t)c * rst] = x; });
}

// the warp's sum of v (harmonics 32 w .. 32 w + 31) into its own slot of the corrector's
// partials: the sums reach k_cgce_sums in a fixed order, so the corrector norm -- and the
// timestep the norm controls -- are the same bits on every run
__device__ __forceinline__ void warp_partial(double v, const StepArgs& a, int slot) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if ((threadIdx.x & 31) == 0 && w < a.nwarp) a.cpart[(size_t)slot * a.nwarp + w] = v;  // w >= nwarp: no harmonic
}

// red[s] = the sum of the per-warp partials of slot s; one warp per slot, lanes over the
// warps in a fixed stride, then a fixed shuffle tree
__global__ void k_cgce_sums(const double* part, int nwarp, double* red) {
  const int s = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double v = 0.0;
  for (int w = lane; w < nwarp; w += 32) v = v + part[(size_t)s * nwarp + w];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) red[s] = v;
}

// Corrector (velocity.F90:413-439, codensity.F90:240-259, magnetic.F90:414-461)
// red[] slots: 0 vTor, 1 vPol, 2 cod, 3 comp, 4 bTor, 5 bicTor, 6 bPol, 7 bicPol.
// The sum of squares of the corrections is accumulated per harmonic in the order the
// back substitution produces them (n decreasing) and across harmonics by atomics.
template <int KL>
__global__ void __launch_bounds__(SOLVE_THREADS) k_corrector(StepArgs a) {
  const int job = blockIdx.y;
  if (job == J_COMP && !a.comp) return;
  if ((job == J_MTOR || job == J_MPOL) && a.Nic > 1) return;  // k_mag_ic
  const int nh = blockIdx.x * blockDim.x + threadIdx.x;
  double ss = 0.0, ssic = 0.0;
  if (nh < a.H) {
    const int l = a.hl[nh], N = a.N, L = a.L;
    const ColView v = col_view<KL>(a, job, nh, l);
    const size_t rst = v.rst;
    const double2 z2 = make_double2(0.0, 0.0);
    const double c = a.implicit;
    // nc = c (N - N_saved) ; N_saved = N ; zerobc (tim_nlincorr, timestep.F90:696-715)
    // vel_setbc_Tor (Re part; velocity.F90:291-299): only no-slip walls (i_vel_bc <= 2)
    const bool tor10 = job == J_VTOR && l == 1 && a.hm[nh] == 0 && a.vel_bc <= 2;
    const double wr = tor10 ? a.rot[ROT_OMEGA] * a.rtor10[0] : 0.0;
    // the right-hand side in W1 (the forward pass then overwrites it row by row, in place)
    diff_terms(v.Nn, v.S, v.W1, rst, N, c);
    auto inC = [&](int n) {
      if (n == 0) return tor10 ? make_double2(wr - v.X[0].x, 0.0) : z2;
      if (n == N - 1) return z2;
      return v.W1[(size_t)n * rst];
    };
    // x += d ; dterr sum of d^2 (tim_addcorr, timestep.F90:717-737)
    auto addcorr = [&](int n, double2 d) {
      const double2 x = v.X[(size_t)n * rst];
      v.X[(size_t)n * rst] = make_double2(x.x + d.x, x.y + d.y);
      ss = ss + d.x * d.x + d.y * d.y;
    };
    auto w1 = [&](int cc, double2 x) { v.W1[(size_t)cc * rst] = x; };
    auto r1 = [&](int n) { return v.W1[(size_t)n * rst]; };
    const bool zero = (job == J_COD || job == J_COMP);
    double2 x0 = z2;
    if (job == J_VPOL) {
      if (l == 0) {
        for (int n = 0; n < N; ++n) addcorr(n, inC(n));
      } else {
        stream_forward<KL>(v.B2, N, inC, w1);
        stream_backward<KL>(v.B2, N, r1, [&](int cc, double2 x) { v.W2[(size_t)cc * rst] = x; });
        auto inD = [&](int n) { return (n == 0 || n == N - 1) ? z2 : v.W2[(size_t)n * rst]; };
        double2 xN = z2;
        stream_forward<KL>(v.B1, N, inD, w1);
        stream_backward<KL>(v.B1, N, r1, [&](int cc, double2 x) {
          v.W2[(size_t)cc * rst] = x;
          if (cc == N - 1) xN = x;
          if (cc == 0) x0 = x;
        });
        double2 ca, cb;
        gre_coeffs(v.iG, x0, xN, ca, cb);
#pragma unroll 8
        for (int n = 0; n < N; ++n) {
          const double g1 = __ldg(v.g + (size_t)(2 * n) * L), g2 = __ldg(v.g + (size_t)(2 * n + 1) * L);
          const double2 x = v.W2[(size_t)n * rst];
          addcorr(n, make_double2(x.x - ca.x * g1 - cb.x * g2, x.y - ca.y * g1 - cb.y * g2));
        }
      }
    } else if (l != 0 || zero) {
      stream_forward<KL>(v.B1, N, inC, w1);
      stream_backward<KL>(v.B1, N, r1, [&](int cc, double2 x) { addcorr(cc, x); if (cc == 0) x0 = x; });
    } else {
      for (int n = 0; n < N; ++n) addcorr(n, inC(n));
    }
    if ((job == J_MTOR || job == J_MPOL) && l != 0) ssic = x0.x * x0.x + x0.y * x0.y;  // inner-core copy (Ni = 1)
  }
  int slot = job == J_VTOR ? 0 : job == J_VPOL ? 1 : job == J_COD ? 2 : job == J_COMP ? 3 : job == J_MTOR ? 4 : 6;
  warp_partial(ss, a, slot);
  if (job == J_MTOR || job == J_MPOL) warp_partial(ssic, a, slot + 1);
}

// The field with a conducting inner core (mag_predictor / mag_corrector, magnetic.F90:370-461;
// tim_icinvX, timestep.F90:594-634).  Each column is one system of NL = Nic + N - 1 unknowns:
// index c < Nic - 1 is the inner core's row c, c >= Nic - 1 the outer core's row c - (Nic - 1)
// (c = Nic - 1, the inner-core boundary, belongs to both).  The inner core's nonlinear term
// -rot_omega d/dphi of its field (nonlinear.F90:451-472) is formed here from the field and
// the rate of the evaluation.  The forward pass keeps its rows in the field's two work
// column sets (2 N >= NL rows).  grid (ceil(H / SOLVE_THREADS), 2): job row 0 toroidal,
// 1 poloidal.  CORR: the corrector (nc = c (N - N_saved), x += correction, dterr sums).
template <int KL, bool CORR>
__global__ void __launch_bounds__(SOLVE_THREADS) k_mag_ic(StepArgs a) {
  const int k = blockIdx.y, job = k == 0 ? J_MTOR : J_MPOL;
  const int nh = blockIdx.x * blockDim.x + threadIdx.x;
  double ss = 0.0, ssic = 0.0;
  if (nh < a.H) {
    const int l = a.hl[nh], N = a.N, L = a.L, Ni = a.Nic, NL = N + Ni - 1;
    const ColView v = col_view<KL>(a, job, nh, l);
    const size_t rst = v.rst;
    const double2 z2 = make_double2(0.0, 0.0);
    const size_t Fi = (size_t)Ni * a.H;
    cplx* icX = a.icstate + (size_t)k * Fi + nh;
    cplx* icS = a.icsv + (size_t)k * Fi + nh;
    const double om = a.rot[ROT_OMEGA_EVAL], m_ = (double)a.hm[nh], c = a.implicit;
    auto icN = [&](int n) {  // -omega (var_coll_dph of the field)
      const double2 x = icX[(size_t)n * rst];
      const double dre = -(x.y * m_), dim = x.x * m_;
      return make_double2(-om * dre, -om * dim);
    };
    // work rows: the outer core's in W1 (row n at cc = n + Nic - 1), the inner core's in W2
    auto wk = [&](int cc) { return cc >= Ni - 1 ? v.W1 + (size_t)(cc - (Ni - 1)) * rst : v.W2 + (size_t)cc * rst; };
    if (!CORR) {
      if (l == 0) {  // not solved: the right-hand sides with their boundary rows
        for (int n = 0; n < Ni; ++n) {
          const double2 x = icN(n);
          icS[(size_t)n * rst] = x;
          icX[(size_t)n * rst] = (n == 0 || n == Ni - 1) ? z2 : x;
        }
        for (int n = 0; n < N; ++n) {
          const double2 x = __ldg(v.Nn + (size_t)n * rst);
          v.S[(size_t)n * rst] = x;
          v.X[(size_t)n * rst] = (n == 0 || n == N - 1) ? z2 : x;
        }
      } else {
        // B := Y B + N (both meshes) ; zerobc ; invX
        for (int n = 0; n < Ni; ++n) icS[(size_t)n * rst] = icN(n);
        save_terms(v.Nn, v.S, rst, N);
        multy_rows<KL>(v.y1, L, v.X, v.Nn, v.W1, rst, N);           // outer core: Y B + N
        multy_rows<KL>(a.icyt + (size_t)k * Ni * (2 * KL + 1) * L + l, L, icX, icS, v.W2, rst, Ni);  // inner
        auto in = [&](int cc) {
          if (cc < Ni - 1) return cc == 0 ? z2 : *wk(cc);
          const int n = cc - (Ni - 1);
          return (n == 0 || n == N - 1) ? z2 : *wk(cc);
        };
        stream_forward<KL>(v.B1, NL, in, [&](int cc, double2 x) { *wk(cc) = x; });
        stream_backward<KL>(v.B1, NL, [&](int cc) { return *wk(cc); }, [&](int cc, double2 x) {
          if (cc <= Ni - 1) icX[(size_t)cc * rst] = x;
          if (cc >= Ni - 1) v.X[(size_t)(cc - (Ni - 1)) * rst] = x;
        });
      }
    } else {
      // the right-hand side c (N - N_saved) of all NL rows in the work rows (the forward
      // pass overwrites it in place); the saves N_saved := N of both cores
      for (int n = 0; n < Ni; ++n) {
        const double2 nn = icN(n), p = icS[(size_t)n * rst];
        icS[(size_t)n * rst] = nn;
        if (n < Ni - 1) *wk(n) = make_double2(c * (nn.x - p.x), c * (nn.y - p.y));
      }
      diff_terms(v.Nn, v.S, v.W1, rst, N, c);
      auto in = [&](int cc) {
        if (cc < Ni - 1) return cc == 0 ? z2 : *wk(cc);
        const int n = cc - (Ni - 1);
        return (n == 0 || n == N - 1) ? z2 : *wk(cc);
      };
      auto add = [&](cplx* X, double2 d) {
        const double2 x = *X;
        *X = make_double2(x.x + d.x, x.y + d.y);
      };
      if (l == 0) {
        for (int cc = 0; cc < NL; ++cc) {
          const double2 d = in(cc);
          if (cc <= Ni - 1) { add(icX + (size_t)cc * rst, d); ssic = ssic + d.x * d.x + d.y * d.y; }
          if (cc >= Ni - 1) { add(v.X + (size_t)(cc - (Ni - 1)) * rst, d); ss = ss + d.x * d.x + d.y * d.y; }
        }
      } else {
        stream_forward<KL>(v.B1, NL, in, [&](int cc, double2 x) { *wk(cc) = x; });
        stream_backward<KL>(v.B1, NL, [&](int cc) { return *wk(cc); }, [&](int cc, double2 d) {
          if (cc <= Ni - 1) { add(icX + (size_t)cc * rst, d); ssic = ssic + d.x * d.x + d.y * d.y; }
          if (cc >= Ni - 1) { add(v.X + (size_t)(cc - (Ni - 1)) * rst, d); ss = ss + d.x * d.x + d.y * d.y; }
        });
      }
    }
  }
  if (CORR) {  // red slots 4 bTor, 5 bicTor, 6 bPol, 7 bicPol
    warp_partial(ss, a, k == 0 ? 4 : 6);
    warp_partial(ssic, a, k == 0 ? 5 : 7);
  }
}

// rot_predictor / rot_corrector (rotation.F90:40-87) with the torques of non_rotation
// (nonlinear.F90:479-538) from k_products' surface sums (np half-rows' pairs after the
// ROT_NSLOT slots, added here in order); one thread.  The rate of the evaluation is kept
// for the inner core's nonlinear term of the solves that follow.
__global__ void k_rot(double* rot, int np, int corr, double inertia, double implicit, double Ph, double vfac,
                      double mfac, int vel_on, int mag_on, int force0) {
  if (threadIdx.x != 0) return;
  const double PI = 3.1415926535897931;
  double sv = 0.0, sm = 0.0;
  for (int h = 0; h < np; ++h) {
    sv = sv + rot[ROT_NSLOT + 2 * h];
    sm = sm + rot[ROT_NSLOT + 2 * h + 1];
  }
  rot[ROT_SUM_VEL] = sv;
  rot[ROT_SUM_MAG] = sm;
  rot[ROT_OMEGA_EVAL] = rot[ROT_OMEGA];
  const double tv = vel_on ? (rot[ROT_SUM_VEL] * 4.0 * PI / Ph) * vfac : 0.0;  // tra_surfintegral's 4 pi / Ph
  const double tm = mag_on ? (rot[ROT_SUM_MAG] * 4.0 * PI / Ph) * mfac : 0.0;
  rot[ROT_VEL] = tv;
  rot[ROT_MAG] = tm;
  if (force0) {
    if (!corr) rot[ROT_OMEGA] = 0.0;
    return;
  }
  const double dt = rot[ROT_DT];
  if (!corr) rot[ROT_OMEGA] = rot[ROT_OMEGA] + (dt / inertia) * (tv + tm);
  else rot[ROT_OMEGA] = rot[ROT_OMEGA] + (dt * implicit / inertia) * ((tv + tm) - (rot[ROT_SV_VEL] + rot[ROT_SV_MAG]));
  rot[ROT_SV_VEL] = tv;
  rot[ROT_SV_MAG] = tm;
}

// Green's functions and influence matrices of the poloidal velocity (velocity.F90:148-168)
// with the streamed solves on the solve-layout factors: thread l carries both unit
// right-hand sides (g1 in .x: 1 at r_i; g2 in .y: 1 at r_o) through XGre, zeroes the
// boundary rows (tim_zerobc) and solves with XPol; the passes work in place on scr [N][L].
template <int KL>
__global__ void k_greens(int N, int NL, int L, const double* lus, const int* ipivs, double2* scr, double* gre,
                         double* gret, double* invg, int* fail) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l < 1 || l >= L) return;
  constexpr int LD = 3 * KL + 1;
  Band bg, bp;
  bg.f = lus + (size_t)OP_VGRE * NL * LD * L + l; bg.piv = ipivs + (size_t)OP_VGRE * NL * L + l;
  bp.f = lus + (size_t)OP_VPOL * NL * LD * L + l; bp.piv = ipivs + (size_t)OP_VPOL * NL * L + l;
  bg.L = bp.L = L; bg.LD = bp.LD = LD;
  double2* w = scr + l;
  const size_t rst = L;
  auto unit = [&](int n) { return make_double2(n == 0 ? 1.0 : 0.0, n == N - 1 ? 1.0 : 0.0); };
  auto rd = [&](int n) { return w[(size_t)n * rst]; };
  auto wr = [&](int n, double2 x) { w[(size_t)n * rst] = x; };
  stream_forward<KL>(bg, N, unit, wr);
  stream_backward<KL>(bg, N, rd, wr);
  w[0] = make_double2(0.0, 0.0);
  w[(size_t)(N - 1) * rst] = make_double2(0.0, 0.0);
  stream_forward<KL>(bp, N, rd, wr);
  stream_backward<KL>(bp, N, rd, wr);
  const double2 x0 = w[0], xN = w[(size_t)(N - 1) * rst];
  double a4[4] = {x0.x, xN.x, x0.y, xN.y};  // invG(i,j) at a4[(i-1)+2(j-1)]
  if (dev_mat_invert(2, a4, 2) != 0) atomicExch(fail, 4);
  for (int k = 0; k < 4; ++k) invg[(size_t)l * 4 + k] = a4[k];
  double* g1 = gre + (size_t)l * 2 * N;
  double* g2 = g1 + N;
  for (int n = 0; n < N; ++n) {
    const double2 g = w[(size_t)n * rst];
    g1[n] = g.x;
    g2[n] = g.y;
    gret[((size_t)n * 2 + 0) * L + l] = g.x;  // [n][2][L] copy for coalesced use in the solves
    gret[((size_t)n * 2 + 1) * L + l] = g.y;
  }
}

// ---- energies: per-(field, category, n) sums of w_lm |a|^2 ----------------------------
// categories: 0 odd (l-m odd), 1 even, 2 m=0 & l even, 3 m=0   (variables.F90:903-957)
// One CTA per (n, field): each thread strides over the harmonics and the CTA reduces in a
// fixed tree, so the sums (and every diagnostic built on them) are the same bits on every
// call for the same state.
constexpr int NORM_THREADS = 256;
__global__ void __launch_bounds__(NORM_THREADS) k_norms(int N, int H, const int* hl, const int* hm,
                                                        const cplx* const* arrs, double* out) {
  const int n = blockIdx.x, k = blockIdx.y;
  const double2* a = arrs[k] + (size_t)n * H;
  double c[4] = {0.0, 0.0, 0.0, 0.0};
  for (int nh = threadIdx.x; nh < H; nh += NORM_THREADS) {
    const int l = hl[nh], m_ = hm[nh];
    double w = 4.0 * 3.1415926535897931 / (double)(2 * l + 1);
    if (m_ != 0) w = 4.0 * w;
    const double2 v = a[nh];
    const double f = w * (v.x * v.x + v.y * v.y);
    c[((l - m_) & 1) ? 0 : 1] += f;
    if (m_ == 0) {
      if ((l & 1) == 0) c[2] += f;
      c[3] += f;
    }
  }
  __shared__ double red[4][NORM_THREADS];
  for (int q = 0; q < 4; ++q) red[q][threadIdx.x] = c[q];
  __syncthreads();
  for (int h = NORM_THREADS / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
      for (int q = 0; q < 4; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[((size_t)k * 4 + threadIdx.x) * N + n] = red[threadIdx.x][0];
}

// ---- batched banded factorisation / solve (LAPACK band storage per matrix) ------------
__global__ void k_factor_batch(int n, int kl, int nmat, double* ab, int* ipiv, int* info) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nmat) return;
  const int ld = 3 * kl + 1;
  info[k] = dev_dgbtf2(n, kl, ab + (size_t)k * ld * n, ld, ipiv + (size_t)k * n);
}
__global__ void k_solve_batch(int n, int kl, const double* ab, const int* ipiv, int nrhs, const int* map, double* b) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs) return;
  const int ld = 3 * kl + 1;
  const int k = map[r];
  const double* A = ab + (size_t)k * ld * n;
  const int* ip = ipiv + (size_t)k * n;
  const int kd = 2 * kl + 1;
  for (int j = 1; j <= n - 1; ++j) {
    int lm = min(kl, n - j);
    int p = ip[j - 1];
    double xj = b[(size_t)(j - 1) * nrhs + r];
    if (p != j) {
      double xp = b[(size_t)(p - 1) * nrhs + r];
      b[(size_t)(p - 1) * nrhs + r] = xj;
      xj = xp;
      b[(size_t)(j - 1) * nrhs + r] = xj;
    }
    double temp = -xj;
    for (int i = 1; i <= lm; ++i) {
      double a = A[(size_t)(kd + i - 1) + (size_t)ld * (j - 1)];
      b[(size_t)(j + i - 1) * nrhs + r] = b[(size_t)(j + i - 1) * nrhs + r] + a * temp;
    }
  }
  const int kk = 2 * kl, kplus1 = kk + 1;
  for (int j = n; j >= 1; --j) {
    double xj = b[(size_t)(j - 1) * nrhs + r] / A[(size_t)(kplus1 - 1) + (size_t)ld * (j - 1)];
    b[(size_t)(j - 1) * nrhs + r] = xj;
    int lo = kplus1 - j;
    for (int i = j - 1; i >= max(1, j - kk); --i) {
      double a = A[(size_t)(lo + i - 1) + (size_t)ld * (j - 1)];
      b[(size_t)(i - 1) * nrhs + r] = b[(size_t)(i - 1) * nrhs + r] - xj * a;
    }
  }
}

SpecArgs spec_args(lsd_ctx* ctx) {
  SpecArgs a;
  a.N = ctx->N; a.H = ctx->H; a.KL = ctx->KL; a.L = ctx->L;
  a.hl = ctx->d_l; a.r = ctx->d_r; a.r1dr = ctx->d_r1dr; a.dr1 = ctx->d_dr;
  return a;
}

StepArgs step_args(lsd_ctx* ctx) {
  StepArgs a;
  a.N = ctx->N; a.H = ctx->H; a.KL = ctx->KL; a.L = ctx->L;
  a.hl = ctx->d_l; a.hm = ctx->d_m;
  a.lus = ctx->d_lus; a.ipivs = ctx->d_ipivs; a.yt = ctx->d_yt;
  a.gret = ctx->d_gret; a.invg = ctx->d_invg;
  a.state = ctx->d_state; a.nl = ctx->d_nl; a.sv = ctx->d_sv;
  a.work = ctx->d_spec;
  a.implicit = ctx->cfg.implicit;
  a.cod_bc = ctx->cfg.cod_bc; a.comp_bc = ctx->cfg.comp_bc; a.vel_bc = ctx->cfg.vel_bc;
  a.qi = ctx->cfg.qi; a.qo = ctx->cfg.qo; a.qi_comp = ctx->cfg.qi_comp; a.qo_comp = ctx->cfg.qo_comp;
  a.comp = ctx->cfg.comp_tstep;
  a.red = ctx->d_red;
  a.cpart = ctx->d_cpart; a.nwarp = (ctx->H + 31) / 32;
  a.NL = ctx->NL; a.Nic = ctx->Nic;
  a.icstate = ctx->d_icstate; a.icsv = ctx->d_icsv; a.icyt = ctx->d_icyt;
  a.rot = ctx->d_rot;
  a.rtor10 = ctx->d_r + (size_t)(3 + (ctx->nh_l1m0 >= 0 && ctx->nh_l1m0 <= 3 ? ctx->nh_l1m0 : 1)) * ctx->N;
  return a;
}

}  // namespace

// One nonlinear evaluation: main.F90:102-124 for Boussinesq MHD + codensity.
int lsd_eval(lsd_ctx* ctx) { return lsd_eval_marked(ctx, nullptr); }

namespace {
// the evaluation's branch streams of ctx->stream (created on first use), or null
lsd_ctx::Aux* eval_aux(lsd_ctx* ctx) {
  for (lsd_ctx::Aux& x : ctx->eval_aux)
    if (x.origin == ctx->stream) return &x;
  lsd_ctx::Aux x{};
  x.origin = ctx->stream;
  bool ok = cudaEventCreateWithFlags(&x.fork, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < 2 && ok; ++i)
    ok = cudaStreamCreateWithFlags(&x.s[i], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&x.join[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    for (int i = 0; i < 2; ++i) {
      if (x.s[i]) cudaStreamDestroy(x.s[i]);
      if (x.join[i]) cudaEventDestroy(x.join[i]);
    }
    if (x.fork) cudaEventDestroy(x.fork);
    return nullptr;
  }
  ctx->eval_aux.push_back(x);  // the pointer below is used before the next push
  return &ctx->eval_aux.back();
}
}  // namespace

// marks (optional): 5 events recorded after the spectral preparation, the synthesis, the
// FFT+products, the analysis and the tail
int lsd_eval_marked(lsd_ctx* ctx, cudaEvent_t* marks) {
  const size_t F = (size_t)ctx->N * ctx->H;
  const size_t FF = (size_t)ctx->N * ctx->HB * ctx->NM * 4;
  cplx* sp = ctx->d_spec;
  cplx* st = ctx->d_state;
  SpecArgs sa = spec_args(ctx);
  dim3 g(ceil_div(ctx->H, 128), ctx->N);
  cudaStream_t s = ctx->stream;
  const bool anel = ctx->cfg.boussinesq == 0;
  if (ctx->cfg.vel_bc == 4) {  // main.F90:101
    k_angmom<<<1, 128, 0, s>>>(ctx->N, ctx->H, ctx->nh_l1m0, ctx->nh_l1m1, ctx->d_r,
                               anel ? ctx->d_wts : ctx->d_intr2dr, anel ? 1 : 0, st + LSD_VEL_TOR * F);
    ctx->launches++;
  }
  // three independent chains on forked branches: u (q, s, t and curl) on s, B on branch 0,
  // the codensity (and composition) derivatives on branch 1; joined before the synthesis
  lsd_ctx::Aux* x = eval_aux(ctx);
  if (!x) return lsd_fail(ctx, LSD_ECUDA, "evaluation: branch streams");
  CUDA_TRY(cudaEventRecord(x->fork, s));
  for (int i = 0; i < 2; ++i) CUDA_TRY(cudaStreamWaitEvent(x->s[i], x->fork, 0));
  k_qst<<<g, 128, 0, s>>>(sa, anel ? ctx->d_compr1dr : ctx->d_r1dr, st + LSD_VEL_TOR * F, st + LSD_VEL_POL * F,
                          sp + S_VQ * F, sp + S_VS * F, sp + S_VT * F);
  k_curl<<<g, 128, 0, s>>>(sa, sp + S_VQ * F, sp + S_VS * F, sp + S_VT * F, sp + S_VCQ * F, sp + S_VCS * F, sp + S_VCT * F);
  k_qst<<<g, 128, 0, x->s[0]>>>(sa, ctx->d_r1dr, st + LSD_MAG_TOR * F, st + LSD_MAG_POL * F, sp + S_BQ * F,
                                sp + S_BS * F, sp + S_BT * F);
  k_curl<<<g, 128, 0, x->s[0]>>>(sa, sp + S_BQ * F, sp + S_BS * F, sp + S_BT * F, sp + S_BCQ * F, sp + S_BCS * F,
                                 sp + S_BCT * F);
  k_drC<<<g, 128, 0, x->s[1]>>>(sa, st + LSD_COD_C * F, sp + S_DC * F);
  ctx->launches += 5;
  const bool comp = ctx->cfg.comp_tstep != 0;
  if (comp) {  // comp_transform (composition.F90:196-212)
    k_drC<<<g, 128, 0, x->s[1]>>>(sa, st + LSD_COMP_C * F, sp + S_DCOMP * F);
    ctx->launches++;
  }
  for (int i = 0; i < 2; ++i) {
    CUDA_TRY(cudaEventRecord(x->join[i], x->s[i]));
    CUDA_TRY(cudaStreamWaitEvent(s, x->join[i], 0));
  }
  if (anel) {  // dr q, dr s, dr t (var_coll_TorPol2qstderiv, variables.F90:610-660)
    for (int k = 0; k < 3; ++k) k_drC<<<g, 128, 0, s>>>(sa, sp + (S_VQ + k) * F, sp + (S_VDQ + k) * F);
    ctx->launches += 3;
  }
  if (marks) cudaEventRecord(marks[0], s);
  cplx* fo = ctx->d_four;
  SynthGroup sg[7];
  const int vin[4][3] = {{S_VQ, S_VS, S_VT}, {S_VCQ, S_VCS, S_VCT}, {S_BQ, S_BS, S_BT}, {S_BCQ, S_BCS, S_BCT}};
  for (int i = 0; i < 4; ++i) {
    sg[i].kind = SK_VECTOR;
    for (int k = 0; k < 3; ++k) { sg[i].in[k] = sp + vin[i][k] * F; sg[i].out[k] = fo + (3 * i + k) * FF; }
  }
  sg[4].kind = SK_GRAD3;
  sg[4].in[0] = sp + S_DC * F; sg[4].in[1] = st + LSD_COD_C * F; sg[4].in[2] = nullptr;
  for (int k = 0; k < 3; ++k) sg[4].out[k] = fo + (12 + k) * FF;
  sg[5].kind = SK_GRAD3;
  sg[5].in[0] = sp + S_DCOMP * F; sg[5].in[1] = st + LSD_COMP_C * F; sg[5].in[2] = nullptr;
  for (int k = 0; k < 3; ++k) sg[5].out[k] = fo + (15 + k) * FF;
  int nsyn = comp ? 18 : 15;  // synthesised fields (FFT layout)
  int ng = comp ? 6 : 5;
  if (anel) {  // dr u_r, dr u_th, dr u_ph: tra_qst2rtp of (dr q, dr s, dr t) (transform.fftw3.F90:611-714)
    SynthGroup& d = sg[ng++];
    d.kind = SK_VECTOR;
    for (int k = 0; k < 3; ++k) { d.in[k] = sp + (S_VDQ + k) * F; d.out[k] = fo + (nsyn + k) * FF; }
    nsyn += 3;
  }
  int rc;
  if ((rc = lsd_launch_synth(ctx, sg, ng))) return rc;
  if (marks) cudaEventRecord(marks[1], s);
  cplx* fa = fo + nsyn * FF;  // the 7 (8) product fields, in the analysis layout
  const bool vardt = ctx->cfg.timestep < 0;
  if (vardt) CUDA_TRY(cudaMemsetAsync(ctx->d_cfl, 0, sizeof(double) * 2 * ctx->N, s));
  if (ctx->cfg.rot_tstep) CUDA_TRY(cudaMemsetAsync(ctx->d_rot + ROT_NSLOT, 0, sizeof(double) * 4 * ctx->HB, s));
  if ((rc = lsd_launch_products(ctx, fo, fa))) return rc;
  if (vardt && (rc = lsd_launch_cfl_finish(ctx))) return rc;  // non_maxtstep
  if (marks) cudaEventRecord(marks[2], s);
  AnalGroup ag[4];
  ag[0].kind = AK_VECTOR;
  ag[1].kind = AK_VECTOR;
  ag[2].kind = AK_SCALAR;
  for (int k = 0; k < 3; ++k) {
    ag[0].in[k] = fa + k * FF; ag[0].out[k] = sp + (S_VQ + k) * F;
    ag[1].in[k] = fa + (3 + k) * FF; ag[1].out[k] = sp + (S_BQ + k) * F;
  }
  ag[2].in[0] = fa + 6 * FF; ag[2].out[0] = sp + S_DC * F;
  ag[2].in[1] = ag[2].in[2] = nullptr; ag[2].out[1] = ag[2].out[2] = nullptr;
  ag[3].kind = AK_SCALAR;
  ag[3].in[0] = fa + 7 * FF; ag[3].out[0] = sp + S_DCOMP * F;
  ag[3].in[1] = ag[3].in[2] = nullptr; ag[3].out[1] = ag[3].out[2] = nullptr;
  if ((rc = lsd_launch_anal(ctx, ag, comp ? 4 : 3))) return rc;
  if (marks) cudaEventRecord(marks[3], s);
  TailArgs ta;
  ta.s = sa;
  ta.dT0 = anel ? ctx->d_ref + (size_t)REF_DT * ctx->N : nullptr;
  const lsd_config& c = ctx->cfg;
  ta.Ra = c.Ra; ta.Ra_comp = c.Ra_comp; ta.Pm2 = c.Pm * c.Pm; ta.Pr = c.Pr; ta.Sc = c.Sc;
  ta.source = c.source; ta.source_comp = c.source_comp;
  ta.vq = sp + S_VQ * F; ta.vs = sp + S_VS * F; ta.vt = sp + S_VT * F;
  ta.bq = sp + S_BQ * F; ta.bs = sp + S_BS * F; ta.bt = sp + S_BT * F;
  ta.cod = sp + S_DC * F;
  ta.comp = comp ? sp + S_DCOMP * F : nullptr;
  ta.C = st + LSD_COD_C * F;
  ta.Comp = st + LSD_COMP_C * F;
  ta.vNTor = ctx->d_nl + LSD_N_VEL_TOR * F; ta.vNPol = ctx->d_nl + LSD_N_VEL_POL * F;
  ta.bNTor = ctx->d_nl + LSD_N_MAG_TOR * F; ta.bNPol = ctx->d_nl + LSD_N_MAG_POL * F;
  ta.codNC = ctx->d_nl + LSD_N_COD * F;
  ta.compNC = ctx->d_nl + LSD_N_COMP * F;
  k_tail<<<g, 128, 0, s>>>(ta);
  ctx->launches++;
  if (marks) cudaEventRecord(marks[4], s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("evaluation: ") + cudaGetErrorString(e));
  return LSD_OK;
}

namespace {
// threads per CTA: ctx->solve_threads (a multiple of 32, at most SOLVE_THREADS; the
// autotuner's choice); one thread per harmonic whatever the CTA size, so the results and
// the per-warp corrector partials do not depend on it
template <int KL>
void launch_pred(lsd_ctx* ctx, const StepArgs& a, bool corr) {
  const int T = ctx->solve_threads;
  dim3 g(ceil_div(ctx->H, T), J_NJOB);
  if (corr) k_corrector<KL><<<g, T, 0, ctx->stream>>>(a);
  else k_predictor<KL><<<g, T, 0, ctx->stream>>>(a);
  if (ctx->Nic > 1) {  // the field coupled to the inner core
    dim3 gi(ceil_div(ctx->H, T), 2);
    if (corr) k_mag_ic<KL, true><<<gi, T, 0, ctx->stream>>>(a);
    else k_mag_ic<KL, false><<<gi, T, 0, ctx->stream>>>(a);
    ctx->launches++;
  }
}

// rot_predictor / rot_corrector before the solves (main.F90:136, 148)
void launch_rot(lsd_ctx* ctx, bool corr) {
  const lsd_config& c = ctx->cfg;
  if (!c.rot_tstep) return;
  const double ri = c.rratio / (1.0 - c.rratio), r3 = ri * ri * ri;  // mes_oc%r(1,3)
  k_rot<<<1, 32, 0, ctx->stream>>>(ctx->d_rot, 2 * ctx->HB, corr ? 1 : 0, ctx->rot_inertia, c.implicit, (double)ctx->Ph,
                                   r3 * c.Pm, r3 * 2 * c.Pm / c.E, c.vel_bc <= 2 ? 1 : 0, ctx->Nic > 1 ? 1 : 0,
                                   c.rot_force_0);
  ctx->launches++;
}

int launch_step_kernel(lsd_ctx* ctx, const StepArgs& a, bool corr) {
  switch (ctx->KL) {
    case 2: launch_pred<2>(ctx, a, corr); break;
    case 3: launch_pred<3>(ctx, a, corr); break;
    case 4: launch_pred<4>(ctx, a, corr); break;
    case 5: launch_pred<5>(ctx, a, corr); break;
    case 6: launch_pred<6>(ctx, a, corr); break;
    default: return lsd_fail(ctx, LSD_EARG, "stencil half-width KL must be 2..6 for the step kernels");
  }
  return LSD_OK;
}
}  // namespace

int lsd_pred(lsd_ctx* ctx) {
  StepArgs a = step_args(ctx);
  launch_rot(ctx, false);
  int rc = launch_step_kernel(ctx, a, false);
  if (rc) return rc;
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_predictor: ") + cudaGetErrorString(e));
  return LSD_OK;
}

int lsd_corr(lsd_ctx* ctx) {
  StepArgs a = step_args(ctx);
  cudaMemsetAsync(ctx->d_cpart, 0, sizeof(double) * 8 * a.nwarp, ctx->stream);  // slots no job writes
  launch_rot(ctx, true);
  int rc = launch_step_kernel(ctx, a, true);
  if (rc) return rc;
  k_cgce_sums<<<1, 256, 0, ctx->stream>>>(ctx->d_cpart, a.nwarp, ctx->d_red);
  ctx->launches += 2;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_corrector: ") + cudaGetErrorString(e));
  return LSD_OK;
}

namespace {

// The derived fields (q, s, t and curl of velocity and field), their per-(field,
// category, shell) norms written to d_out (48 N doubles; k_norms writes every slot once,
// each a fixed-order tree sum, so nothing needs clearing), and host copies of all that
// the radial sums need.  d_arrs: device room for 12 pointers.
// wts: 5 N (intr2dr, intr2dr_comp, _compS, _magdiss, _veldiss), ref: 7 N.
int energy_partials(lsd_ctx* ctx, const cplx** d_arrs, double* d_out, double* Fh, double* wts, double* cod0,
                    double* bpolN, double* r, double* dr1, double* ref) {
  const int N = ctx->N, H = ctx->H, KL = ctx->KL;
  const size_t F = (size_t)N * H;
  cplx* sp = ctx->d_spec;
  cplx* st = ctx->d_state;
  SpecArgs sa = spec_args(ctx);
  dim3 g(ceil_div(H, 128), N);
  cudaStream_t s = ctx->stream;
  // velocity: the compressible var_coll_TorPol2qst (io.F90:1799); compr1dr == r1dr when xi = 0
  k_qst<<<g, 128, 0, s>>>(sa, ctx->cfg.boussinesq ? ctx->d_r1dr : ctx->d_compr1dr, st + LSD_VEL_TOR * F,
                          st + LSD_VEL_POL * F, sp + 0 * F, sp + 1 * F, sp + 2 * F);
  k_curl<<<g, 128, 0, s>>>(sa, sp + 0 * F, sp + 1 * F, sp + 2 * F, sp + 3 * F, sp + 4 * F, sp + 5 * F);
  k_qst<<<g, 128, 0, s>>>(sa, ctx->d_r1dr, st + LSD_MAG_TOR * F, st + LSD_MAG_POL * F, sp + 6 * F, sp + 7 * F,
                          sp + 8 * F);
  k_curl<<<g, 128, 0, s>>>(sa, sp + 6 * F, sp + 7 * F, sp + 8 * F, sp + 9 * F, sp + 10 * F, sp + 11 * F);
  const cplx* arrs[12];
  for (int k = 0; k < 12; ++k) arrs[k] = sp + k * F;
  CUDA_TRY(cudaMemcpyAsync(d_arrs, arrs, sizeof(arrs), cudaMemcpyHostToDevice, s));
  k_norms<<<dim3(N, 12), NORM_THREADS, 0, s>>>(N, H, ctx->d_l, ctx->d_m, d_arrs, d_out);
  ctx->launches += 5;
  CUDA_TRY(cudaMemcpyAsync(Fh, d_out, sizeof(double) * 48 * N, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(wts, ctx->d_intr2dr, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(wts + N, ctx->d_wts, sizeof(double) * 4 * N, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(ref, ctx->d_ref, sizeof(double) * 7 * N, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(r, ctx->d_r, sizeof(double) * 7 * N, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(dr1, ctx->d_dr, sizeof(double) * (2 * KL + 1) * N, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpy2DAsync(cod0, sizeof(double), st + LSD_COD_C * F, sizeof(cplx) * H, sizeof(double), N,
                             cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(bpolN, st + LSD_MAG_POL * F + (size_t)(N - 1) * H, sizeof(cplx) * 3,
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return LSD_OK;
}

// The radial dot products and the energy combinations, on the host in the reference's order.
int energy_finish(lsd_ctx* ctx, const double* Fh, const double* wts, const double* cod0, const double* bpolN,
                  const double* r, const double* dr1, const double* ref, double* out) {
  const int N = ctx->N, KL = ctx->KL;
  const bool bq = ctx->cfg.boussinesq != 0;
  // radial weights: intr2dr (Boussinesq velocity), intr2dr_comp (anelastic velocity,
  // var_coll_norm_comp), intr2dr_magdiss (ohmic dissipation, var_coll_norm_magdiss)
  const double* wv = bq ? wts : wts + N;
  const double* wm = wts;
  const double* wmd = wts + 3 * N;
  const double* wvd = wts + 4 * N;
  auto normw = [&](int k, const double* w, double& Eo, double& Ee, double& E1, double& E0) {
    double v[4];
    for (int q = 0; q < 4; ++q) {
      double acc = 0.0;
      for (int n = 0; n < N; ++n) acc = acc + Fh[((size_t)k * 4 + q) * N + n] * w[n];
      v[q] = acc;
    }
    Eo = v[0]; Ee = v[1]; E1 = v[2]; E0 = v[3];
  };
  // var_coll_norm_surf: rho r |a|^2 on the walls (r alone for the Boussinesq equations)
  auto surf = [&](int k, int n) {
    double f = Fh[((size_t)k * 4 + 0) * N + n] + Fh[((size_t)k * 4 + 1) * N + n];
    return bq ? f * r[(size_t)4 * N + n] : f * ref[REF_RHO * N + n] * r[(size_t)4 * N + n];
  };
  for (int i = 0; i < LSD_NENERGY; ++i) out[i] = 0.0;
  out[LSD_E_TIME] = ctx->t;
  const lsd_config& c = ctx->cfg;
  // io_write2files prefactors (io.F90:234-247)
  const double KE = 0.5, VD = c.Pm;
  const double ME = bq ? c.Pm / c.E : 0.5 * c.Pm / c.E, OD = bq ? 2.0 * c.Pm / c.E : 1.0 * c.Pm / c.E;
  const int ldm = 2 * KL + 1;
  auto D1 = [&](int row, int col) { return dr1[(size_t)(row - 1) + (size_t)ldm * (col - 1)]; };
  double flx = 0.0;
  for (int j = N - KL; j <= N; ++j) flx = flx - cod0[(size_t)(j - 1)] * D1(KL + 1 + N - j, j);
  const double PI = 3.1415926535897931;
  if (bq) out[LSD_E_TOPFLX] = 4.0 * PI * r[(size_t)5 * N + N - 1] * flx;
  else out[LSD_E_TOPFLX] = 4.0 * PI * r[(size_t)5 * N + N - 1] * ref[REF_RHO * N + N - 1] * ref[REF_T * N + N - 1] * flx;
  flx = 0.0;
  for (int j = 1; j <= 1 + KL; ++j) flx = flx - cod0[(size_t)(j - 1)] * D1(KL + 2 - j, j);
  if (bq) out[LSD_E_BOTFLX] = 4.0 * PI * r[(size_t)5 * N + 0] * flx;
  else out[LSD_E_BOTFLX] = 4.0 * PI * r[(size_t)5 * N + 0] * ref[REF_RHO * N] * ref[REF_T * N] * flx;
  double Eo, Ee, E1, E0;
  {  // velocity: arrays 0..2 q,s,t ; 3..5 curl
    double Ep, Epas, Esym, El1, Et, Etas, EDis, ESin = 0, ESout = 0, Ecomp = 0;
    normw(0, wv, Eo, Ee, E1, E0); Ep = Eo + Ee; Epas = E0; Esym = Ee; El1 = E1;
    if (!bq)  // var_coll_norm_veldiss of q (variables.F90:1034-1061)
      for (int n = 0; n < N; ++n) Ecomp = Ecomp + (Fh[(size_t)0 * N + n] + Fh[(size_t)1 * N + n]) * wvd[n];
    normw(1, wv, Eo, Ee, E1, E0); Ep = Ep + Eo + Ee; Epas = Epas + E0; Esym = Esym + Ee; El1 = El1 + E1;
    normw(2, wv, Eo, Ee, E1, E0); Et = Eo + Ee; Etas = E0; Esym = Esym + Eo; El1 = El1 + E1;
    for (int k = 0; k < 3; ++k) { ESin = ESin + surf(k, 0); ESout = ESout + surf(k, N - 1); }
    normw(3, wv, Eo, Ee, E1, E0); EDis = Eo + Ee;
    normw(4, wv, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    normw(5, wv, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    out[LSD_E_KE] = KE * (Ep + Et);
    out[LSD_E_KE_TOR] = KE * Et;
    out[LSD_E_KE_SYM] = KE * Esym;
    out[LSD_E_KE_L1] = KE * El1;
    out[LSD_E_KE_TM0] = KE * E0;
    out[LSD_E_KE_DIS] = VD * EDis + VD * 2.0 * (ESin - ESout) + Ecomp;
    out[LSD_E_KE_AX] = KE * Epas + KE * Etas;
  }
  {  // magnetic: arrays 6..8, curl 9..11
    double Ep, Epas, Esym, El1, Et, Etas, ETm0, EDis;
    normw(6, wm, Eo, Ee, E1, E0); Ep = Eo + Ee; Epas = E0; Esym = Ee; El1 = E1;
    normw(7, wm, Eo, Ee, E1, E0); Ep = Ep + Eo + Ee; Epas = Epas + E0; Esym = Esym + Ee; El1 = El1 + E1;
    normw(8, wm, Eo, Ee, E1, E0); Et = Eo + Ee; Etas = E0; ETm0 = E0; Esym = Esym + Eo; El1 = El1 + E1;
    normw(9, wmd, Eo, Ee, E1, E0); EDis = Eo + Ee;
    normw(10, wmd, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    normw(11, wmd, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    out[LSD_E_ME] = ME * (Ep + Et);
    out[LSD_E_ME_TOR] = ME * Et;
    out[LSD_E_ME_SYM] = ME * Esym;
    out[LSD_E_ME_L1] = ME * El1;
    out[LSD_E_ME_TM0] = ME * ETm0;
    out[LSD_E_ME_DIS] = OD * EDis;
    out[LSD_E_DIP] = bpolN[2] / r[(size_t)4 * N + N - 1];
    out[LSD_E_QUAD] = 2 * bpolN[4] / r[(size_t)4 * N + N - 1];
    out[LSD_E_ME_AX] = ME * Etas + ME * Epas;
  }
  return LSD_OK;
}

}  // namespace

// Energy diagnostics (io_write_vel_energy io.F90:1739-1926, io_write_mag_energy
// io.F90:1933-2024): device norms, host radial dot products in the reference's order.
int lsd_energy_device(lsd_ctx* ctx, double* out) {
  const int N = ctx->N, KL = ctx->KL;
  std::vector<double> Fh((size_t)48 * N), wts(5 * N), cod0(N), bpolN(3 * 2), r(N * 7), dr1((size_t)(2 * KL + 1) * N),
      ref(7 * N);
  int rc = energy_partials(ctx, (const cplx**)(ctx->d_red + 64), ctx->d_red + 128, Fh.data(), wts.data(),
                           cod0.data(), bpolN.data(), r.data(), dr1.data(), ref.data());
  if (rc) return rc;
  return energy_finish(ctx, Fh.data(), wts.data(), cod0.data(), bpolN.data(), r.data(), dr1.data(), ref.data(), out);
}

// ---- energies with no allocation -------------------------------------------------------
// lsd_energy_static: the energies of lsd_energy_device for callers that must not allocate
// when they ask for diagnostics -- a host code whose device memory is fully committed to
// its state arrays (cudaMalloc would fail), or one that keeps work queued on its stream
// while it writes output (cudaMalloc / cudaFree synchronise the device and would stall that
// pipeline).  The norm partial sums and the 12 field pointers live in a file-scope device
// array instead of context memory; host staging uses the context's pinned buffer, which
// lsd_create sizes for it.  The norm kernel writes every slot of the array once per call
// (a fixed-order tree sum per slot, no atomics), so the previous call's contents are
// simply overwritten and nothing is cleared.  The array is shared by every context on a
// device, so calls that overlap on the GPU (two threads, or two streams) race on it.
// Set-up: each call looks up the array's device address with cudaGetSymbolAddress, with
// the context's device current (the lookup allocates nothing; the first lookup in a
// process may load this module, so make the first call before any stream capture).
namespace {
constexpr int ESTATIC_MAX_N = 1024;  // shells
constexpr int ESTATIC_PTRS = 16;     // 12 field pointers, padded to 128 bytes
}  // namespace
static __device__ __align__(256) double g_energy_scratch[ESTATIC_PTRS + 48 * ESTATIC_MAX_N];  // 384 KiB + 128 B

int lsd_energy_static(lsd_ctx* ctx, double* out) {
  const int N = ctx->N, KL = ctx->KL;
  char msg[160];
  if (N > ESTATIC_MAX_N) {
    snprintf(msg, sizeof(msg), "lsd_energies_static: N = %d shells exceeds the static scratch maximum of %d", N,
             ESTATIC_MAX_N);
    return lsd_fail(ctx, LSD_EARG, msg);
  }
  const size_t stage = (size_t)(48 + 5 + 1 + 7 + 2 * KL + 1 + 7) * N + 6;
  if (sizeof(double) * stage > ctx->h_pin_bytes)
    return lsd_fail(ctx, LSD_EARG, "lsd_energies_static: the context's pinned staging buffer is too small");
  double* dscr = nullptr;  // the array's address on the context's device (current here)
  {
    cudaError_t e = cudaGetSymbolAddress((void**)&dscr, g_energy_scratch);
    if (e != cudaSuccess) {
      snprintf(msg, sizeof(msg), "lsd_energies_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return lsd_fail(ctx, LSD_ECUDA, msg);
    }
  }
  double* Fh = ctx->h_pin;
  double* wts = Fh + (size_t)48 * N;
  double* cod0 = wts + (size_t)5 * N;
  double* bpolN = cod0 + N;
  double* r = bpolN + 6;
  double* dr1 = r + (size_t)7 * N;
  double* ref = dr1 + (size_t)(2 * KL + 1) * N;
  int rc = energy_partials(ctx, (const cplx**)dscr, dscr + ESTATIC_PTRS, Fh, wts, cod0, bpolN, r, dr1, ref);
  if (rc) return rc;
  return energy_finish(ctx, Fh, wts, cod0, bpolN, r, dr1, ref, out);
}

// ---- the other diagnostics of io_write2files ------------------------------------------
namespace {
constexpr int HN_MAX = 12;  // arrays per k_hnorm launch
struct HNormArgs {
  const cplx* a[HN_MAX];
  const double* wt[HN_MAX];
};

// Radially integrated norm of every harmonic (the per-harmonic sums of var_coll_normlm,
// variables.F90:1267-1364): out[k][nh] = sum_n w(l,m) |a_k(n,nh)|^2 wt_k(n), n ascending.
// One thread per harmonic; a warp reads 32 consecutive harmonics of row n of the [n][nh]
// layout, so every load is coalesced and the sum order is the reference's.
__global__ void k_hnorm(int N, int H, const int* __restrict__ hl, const int* __restrict__ hm, HNormArgs p,
                        double* __restrict__ out) {
  const int nh = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (nh >= H) return;
  const int l = hl[nh];
  double w = 4.0 * 3.1415926535897931 / (double)(2 * l + 1);
  if (hm[nh] != 0) w = 4.0 * w;
  const cplx* __restrict__ a = p.a[k];
  const double* __restrict__ wt = p.wt[k];
  double e = 0.0;
  for (int n = 0; n < N; ++n) {
    const double2 v = a[(size_t)n * H + nh];
    e = e + w * (v.x * v.x + v.y * v.y) * wt[n];
  }
  out[(size_t)k * H + nh] = e;
}

// Per-shell sums over the harmonics (io_rad_profile, io.F90:2679-2738) for group g of
// three arrays q, s, t: out[g][0][n] = sum_nh w (|q|^2 + |s|^2), out[g][1][n] = sum_nh w |t|^2.
// One block per (shell, group); strided partial sums, then a fixed-order reduction (the
// result does not depend on scheduling).
constexpr int SS_THREADS = 256;
__global__ void __launch_bounds__(SS_THREADS) k_shell_sums(int N, int H, const int* __restrict__ hl,
                                                           const int* __restrict__ hm, HNormArgs p,
                                                           double* __restrict__ out) {
  const int n = blockIdx.x, g = blockIdx.y;
  const cplx* __restrict__ q = p.a[3 * g] + (size_t)n * H;
  const cplx* __restrict__ s = p.a[3 * g + 1] + (size_t)n * H;
  const cplx* __restrict__ t = p.a[3 * g + 2] + (size_t)n * H;
  double ep = 0.0, et = 0.0;
  for (int nh = threadIdx.x; nh < H; nh += SS_THREADS) {
    double w = 4.0 * 3.1415926535897931 / (double)(2 * hl[nh] + 1);
    if (hm[nh] != 0) w = 4.0 * w;
    const double2 a = q[nh], b = s[nh], c = t[nh];
    ep = ep + (w * (a.x * a.x + a.y * a.y) + w * (b.x * b.x + b.y * b.y));
    et = et + w * (c.x * c.x + c.y * c.y);
  }
  for (int o = 16; o > 0; o >>= 1) {
    ep += __shfl_xor_sync(0xffffffffu, ep, o);
    et += __shfl_xor_sync(0xffffffffu, et, o);
  }
  __shared__ double red[2][SS_THREADS / 32];
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { red[0][warp] = ep; red[1][warp] = et; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < SS_THREADS / 32; ++i) { a = a + red[0][i]; b = b + red[1][i]; }
    out[((size_t)g * 2 + 0) * N + n] = a;
    out[((size_t)g * 2 + 1) * N + n] = b;
  }
}

// row n (1-based) of dr(1) applied to a real column x (var_coll_meshmult of one column)
double dr1_row(const double* dr1, int N, int KL, const double* x, int n) {
  const int ldm = 2 * KL + 1;
  double acc = 0.0;
  for (int j = std::max(1, n - KL); j <= std::min(n + KL, N); ++j)
    acc = acc + dr1[(size_t)(KL + n - j) + (size_t)ldm * (j - 1)] * x[j - 1];
  return acc;
}

// io_write_nussel (io.F90:2158-2243) from the l = 0 column of a buoyancy field
void nusselt(const lsd_config& c, const double* dr1, int N, int KL, const double* col0, double* out) {
  const double T_ri = col0[0], T_ro = col0[N - 1];
  const double dCdr_ri = dr1_row(dr1, N, KL, col0, 1), dCdr_ro = dr1_row(dr1, N, KL, col0, N);
  const double ri = c.rratio / (1 - c.rratio), ro = 1 / (1 - c.rratio);
  const double A = (ri * ro) / (ri - ro);
  double nu_top = 0, nu_bot = 0, nu_flux = 0, nu = 0;
  if (c.cod_bc == 1) {
    nu_bot = dCdr_ri / (A / (ri * ri));
    nu_top = dCdr_ro / (A / (ro * ro));
    nu = nu_top;
  } else if (c.cod_bc == 4) {
    const double DT_cond = 1 / ri - 1 / ro, DT = T_ri - T_ro;
    nu_flux = DT_cond / DT;
    nu = nu_flux;
  }
  const double v[8] = {nu, T_ro, T_ri, dCdr_ri, dCdr_ro, nu_top, nu_bot, nu_flux};
  for (int k = 0; k < 8; ++k) out[k] = v[k];
}
}  // namespace

// The time series, spectra and profiles that io_write2files writes besides the energies
// (io.F90:290-340).  Device: the q, s, t fields of velocity and field, their
// per-harmonic radial integrals (k_hnorm) and per-shell harmonic sums (k_shell_sums);
// host: the sums over l and m, the partitions and the scalars in the reference's order.
int lsd_diagnostics_device(lsd_ctx* ctx, double* sc, double* spec, double* prof) {
  const int N = ctx->N, H = ctx->H, KL = ctx->KL, L = ctx->L, M = ctx->M, Mp = ctx->Mp;
  const size_t F = (size_t)N * H;
  const lsd_config& c = ctx->cfg;
  const bool bq = c.boussinesq != 0, comp = c.comp_tstep != 0;
  cplx* sp = ctx->d_spec;
  cplx* st = ctx->d_state;
  cudaStream_t s = ctx->stream;
  // energies and the category norms of q, s, t (slots 0..11 of the spectral scratch)
  std::vector<double> Fh((size_t)48 * N), wts(5 * N), cod0(N), bpolN(3 * 2), r(N * 7),
      dr1((size_t)(2 * KL + 1) * N), ref(7 * N), en(LSD_NENERGY);
  int rc = energy_partials(ctx, (const cplx**)(ctx->d_red + 64), ctx->d_red + 128, Fh.data(), wts.data(),
                           cod0.data(), bpolN.data(), r.data(), dr1.data(), ref.data());
  if (rc) return rc;
  if ((rc = energy_finish(ctx, Fh.data(), wts.data(), cod0.data(), bpolN.data(), r.data(), dr1.data(), ref.data(),
                          en.data())))
    return rc;
  // the field through the compressible var_coll_TorPol2qst (io_write_cmb, io_rad_profile):
  // slots 12..14 when anelastic; the same arrays as slots 6..8 when xi = 0
  const cplx* mc = sp + 6 * F;
  if (!bq) {
    SpecArgs sa = spec_args(ctx);
    dim3 g(ceil_div(H, 128), N);
    k_qst<<<g, 128, 0, s>>>(sa, ctx->d_compr1dr, st + LSD_MAG_TOR * F, st + LSD_MAG_POL * F, sp + 12 * F,
                            sp + 13 * F, sp + 14 * F);
    ctx->launches++;
    mc = sp + 12 * F;
  }
  // output room: the first free slot of the spectral scratch
  const int slot = bq ? 12 : 15;
  const int K = bq ? 8 : 11;
  if (slot + 1 > ctx->nspec || (size_t)(K * H + 4 * N) > 2 * F)
    return lsd_fail(ctx, LSD_EARG, "lsd_diagnostics: spectral scratch too small");
  double* dout = (double*)(sp + (size_t)slot * F);
  HNormArgs p{};
  const double* w2 = ctx->d_intr2dr;
  for (int k = 0; k < 3; ++k) {
    p.a[k] = sp + k * F;            p.wt[k] = w2;   // velocity q, s, t (compressible)
    p.a[3 + k] = sp + (6 + k) * F;  p.wt[3 + k] = w2;  // field q, s, t (var_coll_TorPol2qst_mag)
    if (!bq) { p.a[8 + k] = sp + k * F; p.wt[8 + k] = ctx->d_wts; }  // velocity, intr2dr_comp
  }
  p.a[6] = st + LSD_COD_C * F;  p.wt[6] = w2;
  p.a[7] = st + LSD_COMP_C * F; p.wt[7] = w2;
  k_hnorm<<<dim3(ceil_div(H, 128), K), 128, 0, s>>>(N, H, ctx->d_l, ctx->d_m, p, dout);
  HNormArgs ps{};
  for (int k = 0; k < 3; ++k) { ps.a[k] = sp + k * F; ps.a[3 + k] = mc + k * F; }
  k_shell_sums<<<dim3(N, 2), SS_THREADS, 0, s>>>(N, H, ctx->d_l, ctx->d_m, ps, dout + (size_t)K * H);
  ctx->launches += 2;
  std::vector<double> hn((size_t)K * H + 4 * N), comp0(N);
  std::vector<cplx> cmb((size_t)2 * H), bpol1(2);
  CUDA_TRY(cudaMemcpyAsync(hn.data(), dout, sizeof(double) * hn.size(), cudaMemcpyDeviceToHost, s));
  for (int k = 0; k < 2; ++k)
    CUDA_TRY(cudaMemcpyAsync(cmb.data() + (size_t)k * H, mc + k * F + (size_t)(N - 1) * H, sizeof(cplx) * H,
                             cudaMemcpyDeviceToHost, s));
  const cplx* polN = st + LSD_MAG_POL * F + (size_t)(N - 1) * H;
  CUDA_TRY(cudaMemcpyAsync(&bpol1[0], polN + std::max(ctx->nh_l1m0, 0), sizeof(cplx), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(&bpol1[1], polN + std::max(ctx->nh_l1m1, 0), sizeof(cplx), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpy2DAsync(comp0.data(), sizeof(double), st + LSD_COMP_C * F, sizeof(cplx) * H, sizeof(double), N,
                             cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("lsd_diagnostics: ") + cudaGetErrorString(e));

  const double PI = 3.1415926535897931;
  const double KE = 0.5, ME = bq ? c.Pm / c.E : 0.5 * c.Pm / c.E;
  for (int i = 0; i < LSD_NDIAG; ++i) sc[i] = 0.0;
  sc[LSD_D_TIME] = ctx->t;
  // per-l / per-m sums of one k_hnorm array (var_coll_normlm), nh ascending
  auto normlm = [&](int k, std::vector<double>& El, std::vector<double>& Em) {
    El.assign(L, 0.0); Em.assign(M, 0.0);
    for (int nh = 0; nh < H; ++nh) {
      const double v = hn[(size_t)k * H + nh];
      El[ctx->hl[nh]] = El[ctx->hl[nh]] + v;
      Em[ctx->hm[nh] / Mp] = Em[ctx->hm[nh] / Mp] + v;
    }
  };
  auto normw = [&](int k, const double* w, double& Eo, double& Ee, double& E1, double& E0) {
    double v[4];
    for (int q = 0; q < 4; ++q) {
      double acc = 0.0;
      for (int n = 0; n < N; ++n) acc = acc + Fh[((size_t)k * 4 + q) * N + n] * w[n];
      v[q] = acc;
    }
    Eo = v[0]; Ee = v[1]; E1 = v[2]; E0 = v[3];
  };
  // ---- vel_partition (io.F90:1800-1921)
  {
    const double* wv = bq ? wts.data() : wts.data() + N;
    double Eo, Ee, E1, E0, Ep, Epes, Epesas, Epas, Et, Etes, Etesas, Etas;
    normw(0, wv, Eo, Ee, E1, E0); Ep = Eo + Ee; Epes = Ee; Epesas = E1; Epas = E0;
    normw(1, wv, Eo, Ee, E1, E0); Ep = Ep + Eo + Ee; Epes = Epes + Ee; Epesas = Epesas + E1; Epas = Epas + E0;
    normw(2, wv, Eo, Ee, E1, E0); Et = Eo + Ee; Etes = Eo; Etesas = E0 - E1; Etas = E0;
    std::vector<double> ETl, ETm, EQl, EQm, ESl, ESm;
    normlm(2, ETl, ETm); normlm(0, EQl, EQm); normlm(1, ESl, ESm);
    double l_Eofl = 0.0;
    for (int i = 1; i < L; ++i) l_Eofl = l_Eofl + i * KE * (ETl[i] + EQl[i] + ESl[i]);
    int lpol = 0;
    double best = -1.0;
    for (int i = 0; i < L; ++i)
      if (EQl[i] + ESl[i] > best) { best = EQl[i] + ESl[i]; lpol = i + 1; }  // maxloc, 1-based
    const double v[10] = {KE * Et, KE * Ep, KE * Etas, KE * Epas, KE * Etes, KE * Epes, KE * Etesas, KE * Epesas,
                          l_Eofl, (double)lpol};
    for (int k = 0; k < 10; ++k) sc[LSD_D_VPART + k] = v[k];
  }
  // ---- mag_partition (io.F90:1959-2020)
  {
    const double* wm = wts.data();
    double Eo, Ee, E1, E0, Ep, Epes, Epesas, Epas, Et, Etes, Etesas, Etas;
    normw(6, wm, Eo, Ee, E1, E0); Ep = Eo + Ee; Epes = Ee; Epesas = E1; Epas = E0;
    normw(7, wm, Eo, Ee, E1, E0); Ep = Ep + Eo + Ee; Epes = Epes + Ee; Epesas = Epesas + E1; Epas = Epas + E0;
    normw(8, wm, Eo, Ee, E1, E0); Et = Eo + Ee; Etes = Eo; Etesas = E0 - E1; Etas = E0;
    const double v[8] = {ME * Et, ME * Ep, ME * Etas, ME * Epas, ME * Etes, ME * Epes, ME * Etesas, ME * Epesas};
    for (int k = 0; k < 8; ++k) sc[LSD_D_MPART + k] = v[k];
  }
  // ---- the inner core's field (io_write_mag_energy on mag_icTor / icPol, io.F90:315): q, s,
  // t and curl on its own mesh (spectral slots 0..5, free once the outer core's sums are on
  // the host), category norms per shell, radial sums here; the outer core's Dip / Quad.
  // The call leaves io_MagEn / io_OhmDiss at the inner core's values for dyn_outputs.
  double icE = 0.0, icEDis = 0.0;
  if (ctx->Nic > 1) {
    const int Ni = ctx->Nic;
    const size_t Fi = (size_t)Ni * H;
    SpecArgs si;
    si.N = Ni; si.H = H; si.KL = KL; si.L = L; si.hl = ctx->d_l;
    si.r = ctx->d_icr; si.r1dr = ctx->d_icr1dr; si.dr1 = ctx->d_icdr;
    dim3 gi(ceil_div(H, 128), Ni);
    k_qst<<<gi, 128, 0, s>>>(si, ctx->d_icr1dr, ctx->d_icstate, ctx->d_icstate + Fi, sp, sp + F, sp + 2 * F);
    k_curl<<<gi, 128, 0, s>>>(si, sp, sp + F, sp + 2 * F, sp + 3 * F, sp + 4 * F, sp + 5 * F);
    const cplx* arrs[6];
    for (int k = 0; k < 6; ++k) arrs[k] = sp + k * F;
    const cplx** d_arrs = (const cplx**)(ctx->d_red + 64);
    double* d_out = ctx->d_red + 128;
    CUDA_TRY(cudaMemcpyAsync(d_arrs, arrs, sizeof(arrs), cudaMemcpyHostToDevice, s));
    k_norms<<<dim3(Ni, 6), NORM_THREADS, 0, s>>>(Ni, H, ctx->d_l, ctx->d_m, d_arrs, d_out);
    ctx->launches += 3;
    std::vector<double> Fi_h((size_t)24 * Ni), wic((size_t)5 * Ni);
    CUDA_TRY(cudaMemcpyAsync(Fi_h.data(), d_out, sizeof(double) * Fi_h.size(), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(wic.data(), ctx->d_icintr2dr, sizeof(double) * Ni, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(wic.data() + Ni, ctx->d_icwts, sizeof(double) * 4 * Ni, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    auto nw = [&](int k, const double* w, double& Eo, double& Ee, double& E1, double& E0) {
      double v4[4];
      for (int q = 0; q < 4; ++q) {
        double acc = 0.0;
        for (int n = 0; n < Ni; ++n) acc = acc + Fi_h[((size_t)k * 4 + q) * Ni + n] * w[n];
        v4[q] = acc;
      }
      Eo = v4[0]; Ee = v4[1]; E1 = v4[2]; E0 = v4[3];
    };
    const double* w2i = wic.data();
    const double* wmd = wic.data() + 3 * Ni;  // intr2dr_magdiss of the inner core's mesh
    const double OD = bq ? 2.0 * c.Pm / c.E : 1.0 * c.Pm / c.E;
    double Eo, Ee, E1, E0, Ep, Epes, Epesas, Epas, Et, Etes, Etesas, Etas, Esym, El1, ETm0, EDis;
    nw(0, w2i, Eo, Ee, E1, E0); Ep = Eo + Ee; Epes = Ee; Epesas = E1; Epas = E0; Esym = Ee; El1 = E1;
    nw(1, w2i, Eo, Ee, E1, E0);
    Ep = Ep + Eo + Ee; Epes = Epes + Ee; Epesas = Epesas + E1; Epas = Epas + E0; Esym = Esym + Ee; El1 = El1 + E1;
    nw(2, w2i, Eo, Ee, E1, E0);
    Et = Eo + Ee; Etes = Eo; Etesas = E0 - E1; Etas = E0; ETm0 = E0; Esym = Esym + Eo; El1 = El1 + E1;
    nw(3, wmd, Eo, Ee, E1, E0); EDis = Eo + Ee;
    nw(4, wmd, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    nw(5, wmd, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    icE = ME * (Ep + Et);
    icEDis = OD * EDis;
    const double v9[9] = {icE, ME * Et, ME * Esym, ME * El1, ME * ETm0, icEDis, en[LSD_E_DIP], en[LSD_E_QUAD],
                          ME * Etas + ME * Epas};
    for (int k = 0; k < 9; ++k) sc[LSD_D_MIC + k] = v9[k];
    const double v8[8] = {ME * Et, ME * Ep, ME * Etas, ME * Epas, ME * Etes, ME * Epes, ME * Etesas, ME * Epesas};
    for (int k = 0; k < 8; ++k) sc[LSD_D_MICPART + k] = v8[k];
  }
  {  // rot_torque.dat
    double rot[ROT_NSLOT];  // after the work queued on the context's stream
    CUDA_TRY(cudaMemcpyAsync(rot, ctx->d_rot, sizeof(rot), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    sc[LSD_D_ROT + 0] = rot[ROT_OMEGA]; sc[LSD_D_ROT + 1] = rot[ROT_VEL]; sc[LSD_D_ROT + 2] = rot[ROT_MAG];
  }
  // ---- mag_cmb (io.F90:2036-2145): var_coll_norm_orig of q, s zeroed below the outer shell
  double fdip, thdip;
  {
    double EPol = 0, ESym = 0, El1 = 0, Epas = 0, El12 = 0;
    const double wN = wts[N - 1];
    for (int k = 0; k < 2; ++k) {
      double Fod = 0, Fev = 0, Fl1 = 0, Fm0 = 0, Fl12 = 0;
      for (int nh = 0; nh < H; ++nh) {
        const int l = ctx->hl[nh], m_ = ctx->hm[nh];
        double w = 4.0 * PI / (double)(2 * l + 1);
        if (m_ != 0) w = 4.0 * w;
        const cplx a = cmb[(size_t)k * H + nh];
        const double f = w * (a.x * a.x + a.y * a.y);
        if (m_ == 0) Fm0 = Fm0 + f;
        if (l > 0 && l <= 12) Fl12 = Fl12 + f;
        if (l == 1) Fl1 = Fl1 + f;
        if (((l - m_) % 2 + 2) % 2 == 1) Fod = Fod + f; else Fev = Fev + f;
      }
      EPol = EPol + Fod * wN + Fev * wN;
      ESym = ESym + Fev * wN;
      El1 = El1 + Fl1 * wN;
      Epas = Epas + Fm0 * wN;
      El12 = El12 + Fl12 * wN;
    }
    const double fac = r[(size_t)5 * N + N - 1] / wN;  // r(N,2) / intr2dr(N)
    EPol = ME * EPol * fac; Epas = ME * Epas * fac; ESym = ME * ESym * fac; El1 = ME * El1 * fac;
    El12 = ME * El12 * fac;
    const double g10 = ctx->nh_l1m0 >= 0 ? bpol1[0].x : 0.0;
    double th, ph;
    if (Mp == 1 && M > 1 && ctx->nh_l1m1 >= 0) {
      const double g11 = -2.0 * bpol1[1].x, h11 = 2.0 * bpol1[1].y;
      th = std::sqrt(g10 * g10 + g11 * g11 + h11 * h11);
      if (th != 0.0) th = std::acos(g10 / std::max(th, std::fabs(g10)));
      if (std::fabs(g11) < 1e-99) {
        ph = h11 >= 0.0 ? 0.5 * PI : 1.5 * PI;
      } else {
        ph = std::atan(h11 / g11);
        if (g11 < 0.0) ph = ph + PI;
        if (ph < 0.0) ph = ph + 2.0 * PI;
      }
    } else {
      th = g10 >= 0.0 ? 0.0 : PI;
      ph = 0.0;
    }
    fdip = std::sqrt(El1 / El12);
    thdip = th;
    const double v[7] = {EPol, ESym, El1, th, ph, Epas, El12};
    for (int k = 0; k < 7; ++k) sc[LSD_D_CMB + k] = v[k];
  }
  // ---- Nusselt numbers
  nusselt(c, dr1.data(), N, KL, cod0.data(), sc + LSD_D_NUSC);
  if (comp) nusselt(c, dr1.data(), N, KL, comp0.data(), sc + LSD_D_NUSX);
  // ---- dyn_outputs (io.F90:2355-2399; io_vol io.F90:76)
  {
    const double ri = c.rratio / (1 - c.rratio), ro = 1 / (1 - c.rratio);
    const double vol = (4.0 / 3.0 * PI) * (ro * ro * ro - ri * ri * ri);
    const double Kin = en[LSD_E_KE], Visc = en[LSD_E_KE_DIS];
    const double Mag = ctx->Nic > 1 ? icE : en[LSD_E_ME], Ohm = ctx->Nic > 1 ? icEDis : en[LSD_E_ME_DIS];
    const double Rm = std::sqrt((2 * Kin) / vol), Re = Rm / c.Pm;
    const double El = (c.E * Mag) / (c.Pm * vol);
    const double Le = std::sqrt((2 * c.E * c.E * Mag) / (c.Pm * c.Pm * vol));
    const double v[13] = {Rm, Re, Re * c.Pr, Re * c.Sc, Re * c.E, Mag / Kin, El, Le, fdip, Ohm / (Ohm + Visc),
                          thdip, sc[LSD_D_NUSC], comp ? sc[LSD_D_NUSX] : 0.0};
    for (int k = 0; k < 13; ++k) sc[LSD_D_DYN + k] = v[k];
  }
  sc[LSD_D_DT + 0] = ctx->dt;
  sc[LSD_D_DT + 1] = ctx->corr_dt;
  sc[LSD_D_DT + 2] = ctx->cfl_dt;
  // ---- spectra (io_save_spectrum / _anelastic / io_save_spectrum1)
  if (spec) {
    double* q = spec;
    auto vec_spec = [&](int k0, double Efac) {
      std::vector<double> ETl, ETm, EQl, EQm, ESl, ESm;
      normlm(k0 + 2, ETl, ETm); normlm(k0, EQl, EQm); normlm(k0 + 1, ESl, ESm);
      for (int l = 0; l < L; ++l) {
        *q++ = Efac * (ETl[l] + EQl[l] + ESl[l]); *q++ = Efac * (EQl[l] + ESl[l]); *q++ = Efac * ETl[l];
      }
      for (int m = 0; m < M; ++m) {
        *q++ = Efac * (ETm[m] + EQm[m] + ESm[m]); *q++ = Efac * (EQm[m] + ESm[m]); *q++ = Efac * ETm[m];
      }
    };
    vec_spec(bq ? 0 : 8, KE);
    vec_spec(3, ME);
    for (int k = 6; k < 8; ++k) {
      std::vector<double> El, Em;
      normlm(k, El, Em);
      for (int l = 0; l < L; ++l) *q++ = El[l];
      for (int m = 0; m < M; ++m) *q++ = Em[m];
    }
  }
  // ---- profiles (io_rad_profile, io_save_profile)
  if (prof) {
    const double* ssum = hn.data() + (size_t)K * H;
    for (int n = 0; n < N; ++n) prof[n] = r[(size_t)4 * N + n];
    for (int g = 0; g < 2; ++g) {
      const double Efac = g == 0 ? KE : ME;
      double* out = prof + (size_t)(1 + 3 * g) * N;
      for (int n = 0; n < N; ++n) {
        out[N + n] = Efac * ssum[((size_t)g * 2 + 0) * N + n];
        out[2 * N + n] = Efac * ssum[((size_t)g * 2 + 1) * N + n];
        out[n] = out[2 * N + n] + out[N + n];
      }
    }
    for (int k = 0; k < 2; ++k) {
      const double* col = k == 0 ? cod0.data() : comp0.data();
      for (int n = 0; n < N; ++n) {
        prof[(size_t)(7 + 2 * k) * N + n] = col[n];
        prof[(size_t)(8 + 2 * k) * N + n] = dr1_row(dr1.data(), N, KL, col, n + 1);
      }
    }
  }
  return LSD_OK;
}

// ---- boundary layout: coll Re/Im (N, H) column-major <-> device [n][nh] complex ---------
namespace {
constexpr int TT = 32;  // transpose tile
__global__ void k_coll_to_state(int N, int H, const double* __restrict__ re, const double* __restrict__ im,
                                cplx* __restrict__ out) {
  __shared__ double2 t[TT][TT + 1];
  const int nh0 = blockIdx.x * TT, n0 = blockIdx.y * TT;
  for (int i = threadIdx.y; i < TT; i += blockDim.y) {  // read along n (contiguous in coll)
    const int nh = nh0 + i, n = n0 + threadIdx.x;
    if (nh < H && n < N) t[i][threadIdx.x] = make_double2(re[(size_t)nh * N + n], im[(size_t)nh * N + n]);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < TT; i += blockDim.y) {  // write along nh
    const int n = n0 + i, nh = nh0 + threadIdx.x;
    if (nh < H && n < N) out[(size_t)n * H + nh] = t[threadIdx.x][i];
  }
}
__global__ void k_state_to_coll(int N, int H, const cplx* __restrict__ in, double* __restrict__ re,
                                double* __restrict__ im) {
  __shared__ double2 t[TT][TT + 1];
  const int nh0 = blockIdx.x * TT, n0 = blockIdx.y * TT;
  for (int i = threadIdx.y; i < TT; i += blockDim.y) {
    const int n = n0 + i, nh = nh0 + threadIdx.x;
    if (nh < H && n < N) t[threadIdx.x][i] = in[(size_t)n * H + nh];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < TT; i += blockDim.y) {
    const int nh = nh0 + i, n = n0 + threadIdx.x;
    if (nh < H && n < N) {
      const double2 v = t[i][threadIdx.x];
      re[(size_t)nh * N + n] = v.x;
      im[(size_t)nh * N + n] = v.y;
    }
  }
}
}  // namespace

int lsd_launch_greens(lsd_ctx* ctx, int* d_fail) {
  const int N = ctx->N, NL = ctx->NL, L = ctx->L;
  const int g = ceil_div(L, 32);
  double2* scr = ctx->d_grescr;
  cudaStream_t s = ctx->stream;
  switch (ctx->KL) {
    case 2: k_greens<2><<<g, 32, 0, s>>>(N, NL, L, ctx->d_lus, ctx->d_ipivs, scr, ctx->d_gre, ctx->d_gret, ctx->d_invg, d_fail); break;
    case 3: k_greens<3><<<g, 32, 0, s>>>(N, NL, L, ctx->d_lus, ctx->d_ipivs, scr, ctx->d_gre, ctx->d_gret, ctx->d_invg, d_fail); break;
    case 4: k_greens<4><<<g, 32, 0, s>>>(N, NL, L, ctx->d_lus, ctx->d_ipivs, scr, ctx->d_gre, ctx->d_gret, ctx->d_invg, d_fail); break;
    case 5: k_greens<5><<<g, 32, 0, s>>>(N, NL, L, ctx->d_lus, ctx->d_ipivs, scr, ctx->d_gre, ctx->d_gret, ctx->d_invg, d_fail); break;
    case 6: k_greens<6><<<g, 32, 0, s>>>(N, NL, L, ctx->d_lus, ctx->d_ipivs, scr, ctx->d_gre, ctx->d_gret, ctx->d_invg, d_fail); break;
    default: return lsd_fail(ctx, LSD_EARG, "stencil half-width KL must be 2..6 for the step kernels");
  }
  ctx->launches++;
  CUDA_TRY(cudaGetLastError());
  return LSD_OK;
}

int lsd_coll_to_state(lsd_ctx* ctx, const double* re, const double* im, cplx* out) {
  return lsd_coll_to_state_n(ctx, ctx->N, re, im, out);
}
int lsd_state_to_coll(lsd_ctx* ctx, const cplx* in, double* re, double* im) {
  return lsd_state_to_coll_n(ctx, ctx->N, in, re, im);
}
// the same for columns of `rows` radial points (the inner core's Nic)
int lsd_coll_to_state_n(lsd_ctx* ctx, int rows, const double* re, const double* im, cplx* out) {
  dim3 g(ceil_div(ctx->H, TT), ceil_div(rows, TT)), b(TT, 8);
  k_coll_to_state<<<g, b, 0, ctx->stream>>>(rows, ctx->H, re, im, out);
  ctx->launches++;
  CUDA_TRY(cudaGetLastError());
  return LSD_OK;
}
int lsd_state_to_coll_n(lsd_ctx* ctx, int rows, const cplx* in, double* re, double* im) {
  dim3 g(ceil_div(ctx->H, TT), ceil_div(rows, TT)), b(TT, 8);
  k_state_to_coll<<<g, b, 0, ctx->stream>>>(rows, ctx->H, in, re, im);
  ctx->launches++;
  CUDA_TRY(cudaGetLastError());
  return LSD_OK;
}

// ---- the context's operators applied to caller right-hand sides ------------------------
// X_l x = b for every (l, m) column of up to OPS_MAXF fields in one launch (tim_zerobc +
// tim_invX, timestep.F90:566-588, 684-690): codensity / composition (every l), the
// toroidal velocity and the field's toroidal / poloidal scalars (l >= 1; the l = 0 column
// keeps b with zero boundary rows, as tim_invX skips it).  The poloidal velocity is the
// reference's fourth-order composite (velocity.F90:369-395, 445-465 without the Y
// multiply): x = XPol^-1 zerobc(XGre^-1 zerobc(b)), then vel_gre_adjust with the two
// Green's functions so that dx/dr vanishes at both walls.  In place on [N][H] complex
// fields; one thread per harmonic and field, the rows streamed through registers.
constexpr int OPS_MAXF = 8;
struct OpSolveArgs {
  int N, H, L, NL;
  const int* hl;
  const double* lus;
  const int* ipivs;
  const double* gret;
  const double* invg;
  cplx* data;  // nfield consecutive [N][H] fields
  int field[OPS_MAXF];
};

template <int KL>
__global__ void __launch_bounds__(SOLVE_THREADS) k_opsolve(OpSolveArgs a) {
  const int j = blockIdx.y, fld = a.field[j];
  const int nh = blockIdx.x * blockDim.x + threadIdx.x;
  if (nh >= a.H) return;
  const int N = a.N, L = a.L, l = a.hl[nh];
  constexpr int LD = 3 * KL + 1;
  const size_t rst = a.H;
  double2* X = a.data + (size_t)j * N * a.H + nh;
  const double2 z2 = make_double2(0.0, 0.0);
  const bool zero = fld == LSD_COD_C || fld == LSD_COMP_C;
  const int fam = fld == LSD_VEL_TOR ? OP_VTOR : fld == LSD_VEL_POL ? OP_VPOL : fld == LSD_COD_C ? OP_COD
                : fld == LSD_COMP_C ? OP_COMP : fld == LSD_MAG_TOR ? OP_MTOR : OP_MPOL;
  auto band = [&](int f) {
    Band B;
    B.f = a.lus + (size_t)f * a.NL * LD * L + l;
    B.piv = a.ipivs + (size_t)f * a.NL * L + l;
    B.L = L;
    B.LD = LD;
    return B;
  };
  auto in = [&](int n) { return (n == 0 || n == N - 1) ? z2 : X[(size_t)n * rst]; };  // tim_zerobc
  auto rd = [&](int n) { return X[(size_t)n * rst]; };
  auto wr = [&](int c, double2 x) { X[(size_t)c * rst] = x; };
  if (l == 0 && !zero) {
    X[0] = z2;
    X[(size_t)(N - 1) * rst] = z2;
    return;
  }
  const Band B1 = band(fam);
  if (fld == LSD_VEL_POL) {
    const Band B2 = band(OP_VGRE);
    stream_forward<KL>(B2, N, in, wr);
    stream_backward<KL>(B2, N, rd, wr);
    double2 x0 = z2, xN = z2;
    stream_forward<KL>(B1, N, in, wr);
    stream_backward<KL>(B1, N, rd, [&](int c, double2 x) {
      X[(size_t)c * rst] = x;
      if (c == N - 1) xN = x;
      if (c == 0) x0 = x;
    });
    double iG[4];
    for (int i = 0; i < 4; ++i) iG[i] = __ldg(a.invg + (size_t)l * 4 + i);
    double2 ca, cb;
    gre_coeffs(iG, x0, xN, ca, cb);
    const double* g = a.gret + l;
#pragma unroll 8
    for (int n = 0; n < N; ++n) {
      const double g1 = __ldg(g + (size_t)(2 * n) * L), g2 = __ldg(g + (size_t)(2 * n + 1) * L);
      const double2 x = X[(size_t)n * rst];
      X[(size_t)n * rst] = make_double2(x.x - ca.x * g1 - cb.x * g2, x.y - ca.y * g1 - cb.y * g2);
    }
    return;
  }
  stream_forward<KL>(B1, N, in, wr);
  stream_backward<KL>(B1, N, rd, wr);
}

int lsd_operator_solve(lsd_ctx* ctx, int nfield, const int* fields, double* d_data) {
  if (nfield < 1 || nfield > OPS_MAXF) return lsd_fail(ctx, LSD_EARG, "lsd_operator_solve_device: 1..8 fields");
  if (!ctx->have_ops) return lsd_fail(ctx, LSD_ESTATE, "lsd_operator_solve_device: no operators built");
  OpSolveArgs a;
  a.N = ctx->N; a.H = ctx->H; a.L = ctx->L; a.NL = ctx->NL;
  a.hl = ctx->d_l; a.lus = ctx->d_lus; a.ipivs = ctx->d_ipivs; a.gret = ctx->d_gret; a.invg = ctx->d_invg;
  a.data = (cplx*)d_data;
  for (int i = 0; i < OPS_MAXF; ++i) a.field[i] = LSD_COD_C;
  for (int i = 0; i < nfield; ++i) {
    const int f = fields[i];
    if (f < LSD_VEL_TOR || f > LSD_COMP_C)
      return lsd_fail(ctx, LSD_EARG, "lsd_operator_solve_device: field must be one of the five state scalars or composition");
    if ((f == LSD_MAG_TOR || f == LSD_MAG_POL) && ctx->Nic > 1)
      return lsd_fail(ctx, LSD_EARG, "lsd_operator_solve_device: the field's operators are coupled to the inner core (Nic > 1)");
    a.field[i] = f;
  }
  const int T = ctx->solve_threads;
  const dim3 g(ceil_div(ctx->H, T), nfield);
  switch (ctx->KL) {
    case 2: k_opsolve<2><<<g, T, 0, ctx->stream>>>(a); break;
    case 3: k_opsolve<3><<<g, T, 0, ctx->stream>>>(a); break;
    case 4: k_opsolve<4><<<g, T, 0, ctx->stream>>>(a); break;
    case 5: k_opsolve<5><<<g, T, 0, ctx->stream>>>(a); break;
    case 6: k_opsolve<6><<<g, T, 0, ctx->stream>>>(a); break;
    default: return lsd_fail(ctx, LSD_EARG, "stencil half-width KL must be 2..6");
  }
  ctx->launches++;
  CUDA_TRY(cudaGetLastError());
  return LSD_OK;
}

int lsd_factor_batch(lsd_ctx* ctx, int n, int kl, int nmat, double* d_ab, int* d_ipiv, int* d_info) {
  k_factor_batch<<<ceil_div(nmat, 64), 64, 0, ctx->stream>>>(n, kl, nmat, d_ab, d_ipiv, d_info);
  ctx->launches++;
  CUDA_TRY(cudaGetLastError());
  return LSD_OK;
}

int lsd_solve_batch(lsd_ctx* ctx, int n, int kl, int nmat, const double* d_ab, const int* d_ipiv,
                    int nrhs, const int* d_map, double* d_b) {
  (void)nmat;
  k_solve_batch<<<ceil_div(nrhs, 128), 128, 0, ctx->stream>>>(n, kl, d_ab, d_ipiv, nrhs, d_map, d_b);
  ctx->launches++;
  CUDA_TRY(cudaGetLastError());
  return LSD_OK;
}
