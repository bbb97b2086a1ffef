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
#include "lsd_common.cuh"

namespace {

// spectral scratch slots
enum SpecSlot {
  S_VQ = 0, S_VS, S_VT, S_VCQ, S_VCS, S_VCT,
  S_BQ, S_BS, S_BT, S_BCQ, S_BCS, S_BCT,
  S_DC, S_NSPEC_EVAL
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

// q,s,t of a (Tor, Pol) pair: var_coll_TorPol2qst_mag (variables.F90:565-605)
__global__ void k_qst(SpecArgs a, const cplx* tor, const cplx* pol, cplx* q, cplx* s, cplx* t) {
  int nh = blockIdx.x * blockDim.x + threadIdx.x;
  int n = blockIdx.y + 1;
  if (nh >= a.H) return;
  int l = a.hl[nh];
  size_t id = (size_t)(n - 1) * a.H + nh;
  double rm1 = a.r[(size_t)2 * a.N + n - 1];
  double f = ll1d(l) * rm1;
  double2 p = pol[id];
  q[id] = make_double2(p.x * f, p.y * f);
  double2 sv = band_apply(a.r1dr, a.KL, a.N, pol + nh, a.H, n);
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

// Tail of non_velocity / non_magnetic / non_codensity after the analysis:
//   vel: cq += Ra r Pm^2/Pr C (+ comp) ; NTor = qstllcurlr(t) ; NPol = qstllcurlcurlr(q,s)
//   mag: NPol = qstllcurlr(t) ; NTor = qstllcurlcurlr(q,s)
//   cod: NC = analysed scalar, NC(:, nh=0) += source ;  nh = 0 columns zeroed for vel/mag
struct TailArgs {
  SpecArgs s;
  double Ra, Ra_comp, Pm2, Pr, Sc, source;
  const cplx *vq, *vs, *vt, *bq, *bs, *bt, *cod;
  const cplx *C, *Comp;
  cplx *vNTor, *vNPol, *bNTor, *bNPol, *codNC;
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
    // buoyancy d2 = Ra*r*(Pm**2)/Pr (nonlinear.F90:158-185)
    double2 q = a.vq[id];
    double2 c = a.C[id];
    double d2 = a.Ra * r1 * a.Pm2 / a.Pr;
    q.x = q.x + d2 * c.x;
    q.y = q.y + d2 * c.y;
    double2 cm = a.Comp[id];
    double d2c = a.Ra_comp * r1 * a.Pm2 / a.Sc;
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
}

// ---------------------------------------------------------------------------------------
// Column solves.  One thread per harmonic nh; the column x(n) = X[(n-1)*H + nh].
// LU factors in solve layout [N][3KL+1][L], pivots [N][L]; Y bands [N][2KL+1][L].
// ---------------------------------------------------------------------------------------
struct OpView {
  const double* lu;   // [N][3KL+1][L]
  const int* ipiv;    // [N][L]
  const double* y;    // [N][2KL+1][L]
};

__device__ __forceinline__ double luat(const OpView& o, int KL, int L, int row, int col, int l) {
  return o.lu[((size_t)(col - 1) * (3 * KL + 1) + (row - 1)) * L + l];
}

// dgbtrs on a complex column (Re and Im solved with the same real factors)
__device__ void col_lu_solve(const OpView& o, int KL, int L, int N, int l, cplx* x, size_t st) {
  const int kd = 2 * KL + 1;
  for (int j = 1; j <= N - 1; ++j) {
    int lm = min(KL, N - j);
    int p = o.ipiv[(size_t)(j - 1) * L + l];
    double2 xj = x[(size_t)(j - 1) * st];
    if (p != j) {
      double2 xp = x[(size_t)(p - 1) * st];
      x[(size_t)(p - 1) * st] = xj;
      xj = xp;
      x[(size_t)(j - 1) * st] = xj;
    }
    double2 temp = make_double2(-xj.x, -xj.y);
    for (int i = 1; i <= lm; ++i) {
      double a = luat(o, KL, L, kd + i, j, l);
      double2 v = x[(size_t)(j + i - 1) * st];
      v.x = v.x + a * temp.x;
      v.y = v.y + a * temp.y;
      x[(size_t)(j + i - 1) * st] = v;
    }
  }
  const int k = 2 * KL, kplus1 = k + 1;
  for (int j = N; j >= 1; --j) {
    double2 xj = x[(size_t)(j - 1) * st];
    double d = luat(o, KL, L, kplus1, j, l);
    xj.x = xj.x / d;
    xj.y = xj.y / d;
    x[(size_t)(j - 1) * st] = xj;
    int lo = kplus1 - j;
    for (int i = j - 1; i >= max(1, j - k); --i) {
      double a = luat(o, KL, L, lo + i, j, l);
      double2 v = x[(size_t)(i - 1) * st];
      v.x = v.x - xj.x * a;
      v.y = v.y - xj.y * a;
      x[(size_t)(i - 1) * st] = v;
    }
  }
}

// d = Y b + c  (tim_multY, timestep.F90:640-670), written to d (may alias c, not b)
__device__ void col_multY(const OpView& o, int KL, int L, int N, int l, const cplx* b, const cplx* c, cplx* d, size_t st) {
  const int ldm = 2 * KL + 1;
  for (int n = 1; n <= N; ++n) {
    double2 acc = c[(size_t)(n - 1) * st];
    for (int j = max(1, n - KL); j <= min(n + KL, N); ++j) {
      double a = o.y[((size_t)(j - 1) * ldm + (KL + n - j)) * L + l];
      double2 bv = b[(size_t)(j - 1) * st];
      acc.x = acc.x + a * bv.x;
      acc.y = acc.y + a * bv.y;
    }
    d[(size_t)(n - 1) * st] = acc;
  }
}

__device__ __forceinline__ void col_zero_ends(cplx* x, size_t st, int N) {
  x[0] = make_double2(0.0, 0.0);
  x[(size_t)(N - 1) * st] = make_double2(0.0, 0.0);
}

// vel_gre_adjust (velocity.F90:445-465)
__device__ void col_gre_adjust(const double* gre, const double* invg, int N, int l, cplx* x, size_t st) {
  const double* g1 = gre + (size_t)l * 2 * N;
  const double* g2 = g1 + N;
  const double* iG = invg + (size_t)l * 4;
  double2 bi = x[0], bo = x[(size_t)(N - 1) * st];
  double ar = iG[0] * bi.x + iG[2] * bo.x, br = iG[1] * bi.x + iG[3] * bo.x;
  double ai = iG[0] * bi.y + iG[2] * bo.y, bim = iG[1] * bi.y + iG[3] * bo.y;
  for (int n = 0; n < N; ++n) {
    double2 v = x[(size_t)n * st];
    v.x = v.x - ar * g1[n] - br * g2[n];
    v.y = v.y - ai * g1[n] - bim * g2[n];
    x[(size_t)n * st] = v;
  }
}

struct StepArgs {
  int N, H, KL, L;
  const int* hl;
  const int* hm;
  OpView op[OP_NFAM];
  const double* gre;
  const double* invg;
  cplx* state;  // [field][N][H]
  cplx* nl;
  cplx* sv;
  cplx* work;   // [2][N][H] scratch columns
  double implicit;
  int cod_bc, comp_bc;
  double qi, qo, qi_comp, qo_comp;
  int comp;
  double* red;  // corrector: [8] sums of squares
};

// which solve this CTA row performs
enum SolveJob { J_VTOR = 0, J_VPOL, J_COD, J_MTOR, J_MPOL, J_COMP, J_NJOB };

// Predictor (velocity.F90:369-395, codensity.F90:224-234, magnetic.F90:370-408)
__global__ void k_predictor(StepArgs a) {
  int nh = blockIdx.x * blockDim.x + threadIdx.x;
  int job = blockIdx.y;
  if (nh >= a.H) return;
  if (job == J_COMP && !a.comp) return;
  const size_t F = (size_t)a.N * a.H, st = a.H;
  const int l = a.hl[nh], N = a.N, KL = a.KL, L = a.L;
  int fld = 0;
  switch (job) {
    case J_VTOR: fld = LSD_VEL_TOR; break;
    case J_VPOL: fld = LSD_VEL_POL; break;
    case J_COD: fld = LSD_COD_C; break;
    case J_MTOR: fld = LSD_MAG_TOR; break;
    case J_MPOL: fld = LSD_MAG_POL; break;
    case J_COMP: fld = LSD_COMP_C; break;
  }
  cplx* X = a.state + fld * F + nh;
  const cplx* Nn = a.nl + fld * F + nh;
  cplx* S = a.sv + fld * F + nh;
  cplx* W = a.work + (size_t)job * F + nh;
  for (int n = 0; n < N; ++n) S[(size_t)n * st] = Nn[(size_t)n * st];  // save N
  if (job == J_VPOL) {
    // Pol := NPol ; zerobc ; invX(XGre) ; Pol := YPol vel_Pol + Pol ; zerobc ; invX(XPol) ; adjust
    for (int n = 0; n < N; ++n) W[(size_t)n * st] = Nn[(size_t)n * st];
    col_zero_ends(W, st, N);
    if (l != 0) {
      col_lu_solve(a.op[OP_VGRE], KL, L, N, l, W, st);
      col_multY(a.op[OP_VPOL], KL, L, N, l, X, W, W, st);
    }
    col_zero_ends(W, st, N);
    if (l != 0) {
      col_lu_solve(a.op[OP_VPOL], KL, L, N, l, W, st);
      col_gre_adjust(a.gre, a.invg, N, l, W, st);
    }
    for (int n = 0; n < N; ++n) X[(size_t)n * st] = W[(size_t)n * st];
    return;
  }
  const bool zero = (job == J_COD || job == J_COMP);
  const int fam = job == J_VTOR ? OP_VTOR : job == J_COD ? OP_COD : job == J_COMP ? OP_COMP
                : job == J_MTOR ? OP_MTOR : OP_MPOL;
  if (l != 0 || zero) col_multY(a.op[fam], KL, L, N, l, X, Nn, W, st);
  else for (int n = 0; n < N; ++n) W[(size_t)n * st] = Nn[(size_t)n * st];
  col_zero_ends(W, st, N);
  if (zero && nh == 0) {  // cod_setbc / comp_setbc (codensity.F90:126-184)
    int bc = job == J_COD ? a.cod_bc : a.comp_bc;
    double qi = job == J_COD ? a.qi : a.qi_comp, qo = job == J_COD ? a.qo : a.qo_comp;
    if (bc == 1 || bc == 2) W[0].x = 1.0;
    else if (bc == 3 || bc == 4) W[0].x = qi;
    W[(size_t)(N - 1) * st].x = (bc == 2 || bc == 4) ? qo : 0.0;
  }
  // vel_setbc_Tor: l=1, m=0 inner value rot_omega*r_i with rot_omega = 0 -> 0
  if (l != 0 || zero) col_lu_solve(a.op[fam], KL, L, N, l, W, st);
  for (int n = 0; n < N; ++n) X[(size_t)n * st] = W[(size_t)n * st];
}

__device__ __forceinline__ void warp_block_add(double v, double* target) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(target, v);
}

// Corrector (velocity.F90:413-439, codensity.F90:240-259, magnetic.F90:414-461)
// red[] slots: 0 vTor, 1 vPol, 2 cod, 3 comp, 4 bTor, 5 bicTor, 6 bPol, 7 bicPol
__global__ void k_corrector(StepArgs a) {
  int nh = blockIdx.x * blockDim.x + threadIdx.x;
  int job = blockIdx.y;
  bool live = nh < a.H && !(job == J_COMP && !a.comp);
  double ss = 0.0, ssic = 0.0;
  if (live) {
    const size_t F = (size_t)a.N * a.H, st = a.H;
    const int l = a.hl[nh], N = a.N, KL = a.KL, L = a.L;
    int fld = job == J_VTOR ? LSD_VEL_TOR : job == J_VPOL ? LSD_VEL_POL : job == J_COD ? LSD_COD_C
            : job == J_MTOR ? LSD_MAG_TOR : job == J_MPOL ? LSD_MAG_POL : LSD_COMP_C;
    cplx* X = a.state + fld * F + nh;
    const cplx* Nn = a.nl + fld * F + nh;
    cplx* S = a.sv + fld * F + nh;
    cplx* W = a.work + (size_t)job * F + nh;
    const double c = a.implicit;
    for (int n = 0; n < N; ++n) {  // nc = c (N - N_saved) ; N_saved = N
      double2 v = Nn[(size_t)n * st], p = S[(size_t)n * st];
      W[(size_t)n * st] = make_double2(c * (v.x - p.x), c * (v.y - p.y));
      S[(size_t)n * st] = v;
    }
    double2 x0 = X[0];
    col_zero_ends(W, st, N);
    if (job == J_VTOR && l == 1 && a.hm[nh] == 0) W[0].x = 0.0 - x0.x;  // vel_setbc_Tor, tim_it /= 0
    if (job == J_VPOL) {
      if (l != 0) col_lu_solve(a.op[OP_VGRE], KL, L, N, l, W, st);
      col_zero_ends(W, st, N);
      if (l != 0) {
        col_lu_solve(a.op[OP_VPOL], KL, L, N, l, W, st);
        col_gre_adjust(a.gre, a.invg, N, l, W, st);
      }
    } else {
      const bool zero = (job == J_COD || job == J_COMP);
      const int fam = job == J_VTOR ? OP_VTOR : job == J_COD ? OP_COD : job == J_COMP ? OP_COMP
                    : job == J_MTOR ? OP_MTOR : OP_MPOL;
      if (l != 0 || zero) col_lu_solve(a.op[fam], KL, L, N, l, W, st);
    }
    for (int n = 0; n < N; ++n) {  // tim_addcorr
      double2 d = W[(size_t)n * st];
      ss = ss + d.x * d.x;
      ss = ss + d.y * d.y;
      double2 v = X[(size_t)n * st];
      X[(size_t)n * st] = make_double2(v.x + d.x, v.y + d.y);
    }
    if ((job == J_MTOR || job == J_MPOL) && l != 0) {  // inner-core copy (Ni = 1)
      double2 d = W[0];
      ssic = d.x * d.x + d.y * d.y;
    }
  }
  int slot = job == J_VTOR ? 0 : job == J_VPOL ? 1 : job == J_COD ? 2 : job == J_COMP ? 3 : job == J_MTOR ? 4 : 6;
  warp_block_add(ss, a.red + slot);
  if (job == J_MTOR || job == J_MPOL) warp_block_add(ssic, a.red + slot + 1);
}

// ---- energies: per-(field, category, n) partial sums of w_lm |a|^2 ------------------
// categories: 0 odd (l-m odd), 1 even, 2 m=0 & l even, 3 m=0   (variables.F90:903-957)
__global__ void k_norms(int N, int H, const int* hl, const int* hm, const cplx* const* arrs, int narr, double* out) {
  int nh = blockIdx.x * blockDim.x + threadIdx.x;
  int n = blockIdx.y;
  int k = blockIdx.z;
  double f = 0.0;
  int l = 0, m_ = 0;
  if (nh < H) {
    l = hl[nh]; m_ = hm[nh];
    double w = 4.0 * 3.1415926535897931 / (double)(2 * l + 1);
    if (m_ != 0) w = 4.0 * w;
    double2 v = arrs[k][(size_t)n * H + nh];
    f = w * (v.x * v.x + v.y * v.y);
  }
  double c[4];
  c[0] = (nh < H && ((l - m_) % 2 + 2) % 2 == 1) ? f : 0.0;
  c[1] = (nh < H && ((l - m_) % 2 + 2) % 2 == 0) ? f : 0.0;
  c[2] = (nh < H && m_ == 0 && l % 2 == 0) ? f : 0.0;
  c[3] = (nh < H && m_ == 0) ? f : 0.0;
  for (int q = 0; q < 4; ++q) warp_block_add(c[q], out + ((size_t)k * 4 + q) * N + n);
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
  const size_t lus = (size_t)ctx->N * (3 * ctx->KL + 1) * ctx->L;
  const size_t ys = (size_t)ctx->N * (2 * ctx->KL + 1) * ctx->L;
  const size_t ps = (size_t)ctx->N * ctx->L;
  for (int f = 0; f < OP_NFAM; ++f) {
    a.op[f].lu = ctx->d_lus + f * lus;
    a.op[f].ipiv = ctx->d_ipivs + f * ps;
    a.op[f].y = ctx->d_y + f * ys;
  }
  a.gre = ctx->d_gre; a.invg = ctx->d_invg;
  a.state = ctx->d_state; a.nl = ctx->d_nl; a.sv = ctx->d_sv;
  a.work = ctx->d_spec;  // J_NJOB slots of the spectral scratch (free between evaluations)
  a.implicit = ctx->cfg.implicit;
  a.cod_bc = ctx->cfg.cod_bc; a.comp_bc = ctx->cfg.comp_bc;
  a.qi = ctx->cfg.qi; a.qo = ctx->cfg.qo; a.qi_comp = ctx->cfg.qi_comp; a.qo_comp = ctx->cfg.qo_comp;
  a.comp = ctx->cfg.comp_tstep;
  a.red = ctx->d_red;
  return a;
}

}  // namespace

// One nonlinear evaluation: main.F90:102-124 for Boussinesq MHD + codensity.
int lsd_eval(lsd_ctx* ctx) {
  const size_t F = (size_t)ctx->N * ctx->H;
  const size_t FF = (size_t)ctx->N * ctx->NM * ctx->Th;
  cplx* sp = ctx->d_spec;
  cplx* st = ctx->d_state;
  SpecArgs sa = spec_args(ctx);
  dim3 g(ceil_div(ctx->H, 128), ctx->N);
  cudaStream_t s = ctx->stream;
  k_qst<<<g, 128, 0, s>>>(sa, st + LSD_VEL_TOR * F, st + LSD_VEL_POL * F, sp + S_VQ * F, sp + S_VS * F, sp + S_VT * F);
  k_qst<<<g, 128, 0, s>>>(sa, st + LSD_MAG_TOR * F, st + LSD_MAG_POL * F, sp + S_BQ * F, sp + S_BS * F, sp + S_BT * F);
  k_curl<<<g, 128, 0, s>>>(sa, sp + S_VQ * F, sp + S_VS * F, sp + S_VT * F, sp + S_VCQ * F, sp + S_VCS * F, sp + S_VCT * F);
  k_curl<<<g, 128, 0, s>>>(sa, sp + S_BQ * F, sp + S_BS * F, sp + S_BT * F, sp + S_BCQ * F, sp + S_BCS * F, sp + S_BCT * F);
  k_drC<<<g, 128, 0, s>>>(sa, st + LSD_COD_C * F, sp + S_DC * F);
  ctx->launches += 5;
  cplx* fo = ctx->d_four;
  SynthGroup sg[5];
  const int vin[4][3] = {{S_VQ, S_VS, S_VT}, {S_VCQ, S_VCS, S_VCT}, {S_BQ, S_BS, S_BT}, {S_BCQ, S_BCS, S_BCT}};
  for (int i = 0; i < 4; ++i) {
    sg[i].kind = SK_VECTOR;
    for (int k = 0; k < 3; ++k) { sg[i].in[k] = sp + vin[i][k] * F; sg[i].out[k] = fo + (3 * i + k) * FF; }
  }
  sg[4].kind = SK_GRAD3;
  sg[4].in[0] = sp + S_DC * F; sg[4].in[1] = st + LSD_COD_C * F; sg[4].in[2] = nullptr;
  for (int k = 0; k < 3; ++k) sg[4].out[k] = fo + (12 + k) * FF;
  int rc;
  if ((rc = lsd_launch_synth(ctx, sg, 5))) return rc;
  if ((rc = lsd_launch_products(ctx, fo, fo))) return rc;
  AnalGroup ag[3];
  ag[0].kind = AK_VECTOR;
  ag[1].kind = AK_VECTOR;
  ag[2].kind = AK_SCALAR;
  for (int k = 0; k < 3; ++k) {
    ag[0].in[k] = fo + k * FF; ag[0].out[k] = sp + (S_VQ + k) * F;
    ag[1].in[k] = fo + (3 + k) * FF; ag[1].out[k] = sp + (S_BQ + k) * F;
  }
  ag[2].in[0] = fo + 6 * FF; ag[2].out[0] = sp + S_DC * F;
  ag[2].in[1] = ag[2].in[2] = nullptr; ag[2].out[1] = ag[2].out[2] = nullptr;
  if ((rc = lsd_launch_anal(ctx, ag, 3))) return rc;
  TailArgs ta;
  ta.s = sa;
  const lsd_config& c = ctx->cfg;
  ta.Ra = c.Ra; ta.Ra_comp = c.Ra_comp; ta.Pm2 = c.Pm * c.Pm; ta.Pr = c.Pr; ta.Sc = c.Sc;
  ta.source = c.source;
  ta.vq = sp + S_VQ * F; ta.vs = sp + S_VS * F; ta.vt = sp + S_VT * F;
  ta.bq = sp + S_BQ * F; ta.bs = sp + S_BS * F; ta.bt = sp + S_BT * F;
  ta.cod = sp + S_DC * F;
  ta.C = st + LSD_COD_C * F;
  ta.Comp = st + LSD_COMP_C * F;
  ta.vNTor = ctx->d_nl + LSD_N_VEL_TOR * F; ta.vNPol = ctx->d_nl + LSD_N_VEL_POL * F;
  ta.bNTor = ctx->d_nl + LSD_N_MAG_TOR * F; ta.bNPol = ctx->d_nl + LSD_N_MAG_POL * F;
  ta.codNC = ctx->d_nl + LSD_N_COD * F;
  k_tail<<<g, 128, 0, s>>>(ta);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("evaluation: ") + cudaGetErrorString(e));
  return LSD_OK;
}

int lsd_pred(lsd_ctx* ctx) {
  StepArgs a = step_args(ctx);
  dim3 g(ceil_div(ctx->H, 64), J_NJOB);
  k_predictor<<<g, 64, 0, ctx->stream>>>(a);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_predictor: ") + cudaGetErrorString(e));
  return LSD_OK;
}

int lsd_corr(lsd_ctx* ctx) {
  StepArgs a = step_args(ctx);
  cudaMemsetAsync(ctx->d_red, 0, sizeof(double) * 8, ctx->stream);
  dim3 g(ceil_div(ctx->H, 64), J_NJOB);
  k_corrector<<<g, 64, 0, ctx->stream>>>(a);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_corrector: ") + cudaGetErrorString(e));
  return LSD_OK;
}

// Energy diagnostics (io_write_vel_energy io.F90:1739-1926, io_write_mag_energy
// io.F90:1933-2024): device norms, host radial dot products in the reference's order.
int lsd_energy_device(lsd_ctx* ctx, double* out) {
  const int N = ctx->N, H = ctx->H, KL = ctx->KL;
  const size_t F = (size_t)N * H;
  cplx* sp = ctx->d_spec;
  cplx* st = ctx->d_state;
  SpecArgs sa = spec_args(ctx);
  dim3 g(ceil_div(H, 128), N);
  cudaStream_t s = ctx->stream;
  k_qst<<<g, 128, 0, s>>>(sa, st + LSD_VEL_TOR * F, st + LSD_VEL_POL * F, sp + 0 * F, sp + 1 * F, sp + 2 * F);
  k_curl<<<g, 128, 0, s>>>(sa, sp + 0 * F, sp + 1 * F, sp + 2 * F, sp + 3 * F, sp + 4 * F, sp + 5 * F);
  k_qst<<<g, 128, 0, s>>>(sa, st + LSD_MAG_TOR * F, st + LSD_MAG_POL * F, sp + 6 * F, sp + 7 * F, sp + 8 * F);
  k_curl<<<g, 128, 0, s>>>(sa, sp + 6 * F, sp + 7 * F, sp + 8 * F, sp + 9 * F, sp + 10 * F, sp + 11 * F);
  const cplx* arrs[12];
  for (int k = 0; k < 12; ++k) arrs[k] = sp + k * F;
  const cplx** d_arrs = (const cplx**)(ctx->d_red + 64);  // 12 pointers after the sums
  double* d_out = ctx->d_red + 128;
  CUDA_TRY(cudaMemcpyAsync(d_arrs, arrs, sizeof(arrs), cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(double) * 48 * N, s));
  dim3 gn(ceil_div(H, 128), N, 12);
  k_norms<<<gn, 128, 0, s>>>(N, H, ctx->d_l, ctx->d_m, d_arrs, 12, d_out);
  ctx->launches += 5;
  std::vector<double> Fh((size_t)48 * N), wts(N), cod0(N), bpolN(3 * 2), r(N * 7), dr1((size_t)(2 * KL + 1) * N);
  CUDA_TRY(cudaMemcpyAsync(Fh.data(), d_out, sizeof(double) * 48 * N, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(wts.data(), ctx->d_intr2dr, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(r.data(), ctx->d_r, sizeof(double) * 7 * N, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(dr1.data(), ctx->d_dr, sizeof(double) * dr1.size(), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpy2DAsync(cod0.data(), sizeof(double), st + LSD_COD_C * F, sizeof(cplx) * H, sizeof(double), N,
                             cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(bpolN.data(), st + LSD_MAG_POL * F + (size_t)(N - 1) * H, sizeof(cplx) * 3,
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  auto norm = [&](int k, double& Eo, double& Ee, double& E1, double& E0) {
    double v[4];
    for (int q = 0; q < 4; ++q) {
      double acc = 0.0;
      for (int n = 0; n < N; ++n) acc = acc + Fh[((size_t)k * 4 + q) * N + n] * wts[n];
      v[q] = acc;
    }
    Eo = v[0]; Ee = v[1]; E1 = v[2]; E0 = v[3];
  };
  auto surf = [&](int k, int n) { return (Fh[((size_t)k * 4 + 0) * N + n] + Fh[((size_t)k * 4 + 1) * N + n]) * r[(size_t)4 * N + n]; };
  for (int i = 0; i < LSD_NENERGY; ++i) out[i] = 0.0;
  out[LSD_E_TIME] = ctx->t;
  const lsd_config& c = ctx->cfg;
  const double KE = 0.5, VD = c.Pm, ME = c.Pm / c.E, OD = 2.0 * c.Pm / c.E;
  const int ldm = 2 * KL + 1;
  auto D1 = [&](int row, int col) { return dr1[(size_t)(row - 1) + (size_t)ldm * (col - 1)]; };
  double flx = 0.0;
  for (int j = N - KL; j <= N; ++j) flx = flx - cod0[(size_t)(j - 1)] * D1(KL + 1 + N - j, j);
  const double PI = 3.1415926535897931;
  out[LSD_E_TOPFLX] = 4.0 * PI * r[(size_t)5 * N + N - 1] * flx;
  flx = 0.0;
  for (int j = 1; j <= 1 + KL; ++j) flx = flx - cod0[(size_t)(j - 1)] * D1(KL + 2 - j, j);
  out[LSD_E_BOTFLX] = 4.0 * PI * r[(size_t)5 * N + 0] * flx;
  double Eo, Ee, E1, E0;
  {  // velocity: arrays 0..2 q,s,t ; 3..5 curl
    double Ep, Epas, Esym, El1, Et, Etas, EDis, ESin = 0, ESout = 0;
    norm(0, Eo, Ee, E1, E0); Ep = Eo + Ee; Epas = E0; Esym = Ee; El1 = E1;
    norm(1, Eo, Ee, E1, E0); Ep = Ep + Eo + Ee; Epas = Epas + E0; Esym = Esym + Ee; El1 = El1 + E1;
    norm(2, Eo, Ee, E1, E0); Et = Eo + Ee; Etas = E0; Esym = Esym + Eo; El1 = El1 + E1;
    for (int k = 0; k < 3; ++k) { ESin = ESin + surf(k, 0); ESout = ESout + surf(k, N - 1); }
    norm(3, Eo, Ee, E1, E0); EDis = Eo + Ee;
    norm(4, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    norm(5, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    out[LSD_E_KE] = KE * (Ep + Et);
    out[LSD_E_KE_TOR] = KE * Et;
    out[LSD_E_KE_SYM] = KE * Esym;
    out[LSD_E_KE_L1] = KE * El1;
    out[LSD_E_KE_TM0] = KE * E0;
    out[LSD_E_KE_DIS] = VD * EDis + VD * 2.0 * (ESin - ESout);
    out[LSD_E_KE_AX] = KE * Epas + KE * Etas;
  }
  {  // magnetic: arrays 6..8, curl 9..11
    double Ep, Epas, Esym, El1, Et, Etas, ETm0, EDis;
    norm(6, Eo, Ee, E1, E0); Ep = Eo + Ee; Epas = E0; Esym = Ee; El1 = E1;
    norm(7, Eo, Ee, E1, E0); Ep = Ep + Eo + Ee; Epas = Epas + E0; Esym = Esym + Ee; El1 = El1 + E1;
    norm(8, Eo, Ee, E1, E0); Et = Eo + Ee; Etas = E0; ETm0 = E0; Esym = Esym + Eo; El1 = El1 + E1;
    norm(9, Eo, Ee, E1, E0); EDis = Eo + Ee;
    norm(10, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    norm(11, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
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
