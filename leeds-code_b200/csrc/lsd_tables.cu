// lsd_tables.cu -- FP64 device construction of the static tables of one context:
// Gauss-Legendre points and weights (auxiliary/gauwts.f), Schmidt P_l^m and dP/dtheta
// with the derived transform tables (legendre.F90:63-128, auxiliary/schnla.f and helpers),
// the radial Chebyshev grid with finite-difference weights and integration weights
// (meshs.F90:116-419), and the banded time-stepping operators with their LU factors
// (timestep.F90:47-546, velocity.F90:56-273, codensity.F90:37-119, magnetic.F90:62-282).
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "lsd_banded.cuh"
#include "lsd_common.cuh"

namespace {

// ---------------------------------------------------------------------------------------
// Gauss-Legendre nodes on [-1, 1], ascending (gauwts.f:43-71)
// ---------------------------------------------------------------------------------------
__global__ void k_gauss(int nth, double* gp, double* gw, int* fail) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  int m = (nth + 1) / 2;
  if (i > m) return;
  const double EPS = 1.0e-13, PI = 3.14159265358979312;
  const double xm = 0.0, xl = 1.0;  // 0.5*(x2+x1), 0.5*(x2-x1) with x1=-1, x2=1
  double z = cos(PI * ((double)i - 0.25) / ((double)nth + 0.5));
  double z1, pp;
  int iter = 0;
  do {
    double p1 = 1.0, p2 = 0.0, p3;
    for (int j = 1; j <= nth; ++j) {
      p3 = p2; p2 = p1;
      p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / (double)j;
    }
    pp = nth * (z * p1 - p2) / (z * z - 1.0);
    z1 = z;
    z = z1 - p1 / pp;
    if (++iter > 200) { atomicExch(fail, 1); break; }  // bounded Newton loop
  } while (fabs(z - z1) > EPS);
  gp[i - 1] = xm - xl * z;
  gp[nth - i] = xm + xl * z;
  gw[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
  gw[nth - i] = gw[i - 1];
}

__global__ void k_trig(int nth, const double* gp, double* sn, double* sn1) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nth) return;
  double th = acos(gp[j]);
  sn[j] = sin(th);
  sn1[j] = 1.0 / sn[j];
}

// Schmidt helpers (pmm.f, pmm1.f, plm.f, dpmm.f, dpmm1.f, dplm.f)
__device__ double d_pmm(int m, double s) {
  if (m == 0) return 1.0;
  double p = sqrt(2.0);
  for (int i = 1; i <= m; ++i) { double twoi = 2.0 * i; p = p * s * sqrt((twoi - 1.0) / twoi); }
  return p;
}
__device__ double d_dpmm(int m, double c, double s) {
  if (m == 0) return 0.0;
  double d = sqrt(2.0) * (double)m * c / s;
  for (int i = 1; i <= m; ++i) { double twoi = 2.0 * i; d = d * s * sqrt((twoi - 1.0) / twoi); }
  return d;
}

// One thread per (theta point j of the southern half grid, order index m): the
// three-term recurrences in l of schnla.f:66-109 for m_ = m*Mp, then the eight tables.
// Tables are stored [table][nh][Th2] (Fortran leg_*(Th2, 0:H-1)).
__global__ void k_legendre(int L, int M, int Mp, int H, int Th2, const double* gp, const double* gw,
                           const double* sn1, const int* lm2nh, double* leg, int* fail) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int m = blockIdx.y;
  if (j >= Th2 || m >= M) return;
  const double x = gp[j];
  const double sine = sqrt((1.0 + x) * (1.0 - x));
  if (sine < 1.0e-6) { atomicExch(fail, 2); return; }
  const int m_ = m * Mp;
  const size_t T = (size_t)H * Th2;
  double p2 = 0.0, p1 = 0.0, d2 = 0.0, d1 = 0.0;
  for (int l = m_; l < L; ++l) {
    double pa, dpa;
    if (l == m_) {
      pa = d_pmm(m_, sine);
      dpa = d_dpmm(m_, x, sine);
    } else if (l == m_ + 1) {
      pa = x * p1 * sqrt(2.0 * m_ + 1.0);
      dpa = sqrt(2.0 * m_ + 1.0) * (x * d1 - sine * p1);
    } else {
      double rm = m_, rl = l;
      pa = (2.0 * rl - 1.0) * x * p1;
      pa = pa - p2 * sqrt((rl + rm - 1.0) * (rl - rm - 1.0));
      pa = pa / sqrt((rl + rm) * (rl - rm));
      dpa = (2.0 * rl - 1.0) * (x * d1 - sine * p1);
      dpa = dpa - d2 * sqrt((rl + rm - 1.0) * (rl - rm - 1.0));
      dpa = dpa / sqrt((rl + rm) * (rl - rm));
    }
    p2 = p1; p1 = pa; d2 = d1; d1 = dpa;
    int nh = lm2nh[m * L + l];
    if (nh < 0) continue;
    size_t id = (size_t)nh * Th2 + j;
    double s1 = sn1[j];
    leg[LSD_LEG_P * T + id] = pa;
    leg[LSD_LEG_P_ * T + id] = dpa;
    leg[LSD_LEG_SIN1MP * T + id] = pa * m_ * s1;
    double w = gw[j] * ((2.0 * l + 1.0) / 4.0);
    if (m == 0) w = 2.0 * w;
    leg[LSD_LEG_GWP * T + id] = pa * w;
    if (l == 0) {
      leg[LSD_LEG_LLP_ * T + id] = 0.0;
      leg[LSD_LEG_LLSIN1MP * T + id] = 0.0;
      leg[LSD_LEG_GWLLP_ * T + id] = 0.0;
      leg[LSD_LEG_GWLLSIN1MP * T + id] = 0.0;
    } else {
      double w1 = 1.0 / sqrt((double)(l * (l + 1)));
      leg[LSD_LEG_LLP_ * T + id] = dpa * w1;
      leg[LSD_LEG_LLSIN1MP * T + id] = pa * w1 * m_ * s1;
      double w2 = w / sqrt((double)(l * (l + 1)));
      leg[LSD_LEG_GWLLP_ * T + id] = dpa * w2;
      leg[LSD_LEG_GWLLSIN1MP * T + id] = pa * w2 * m_ * s1;
    }
  }
}

// ---------------------------------------------------------------------------------------
// Radial mesh (meshs.F90:135-143, 228-419).  The reference state ref[7][N] (rho, xi,
// dxi/dr, T, dT/dr, eta, deta/dr) is zero with eta = 1 for the Boussinesq equations
// (io.F90:545-556) and the planet model of the anelastic ones (io.F90:559-608).
// ---------------------------------------------------------------------------------------
__global__ void k_grid(int N, double rratio, double alpha, double* r) {
  int n = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (n > N) return;
  const double PI = 3.1415926535897931;
  double x;
  if (alpha > 0)
    x = 0.5 * (1.0 + asin(alpha * cos(PI * (N - n) / (double)(N - 1))) / asin(alpha));
  else
    x = 0.5 * (1.0 + cos(PI * (N - n) / (double)(N - 1)));
  double ri = rratio / (1.0 - rratio);
  x = x + ri;
  for (int p = -3; p <= 3; ++p) {  // integer powers as products, like gfortran's r**p
    double y = 1.0;
    int ap = p < 0 ? -p : p;
    for (int k = 0; k < ap; ++k) y = (k == 0) ? x : y * x;
    r[(size_t)(p + 3) * N + (n - 1)] = p < 0 ? 1.0 / y : (p == 1 ? x : y);
  }
}

// The inner core's mesh (meshs.F90:165-169): r(n) = ri cos(pi (2 Nic - n') / (2 Nic - 1)),
// n' = Nic + n, so that r(Nic) = ri; powers as in k_grid.
__global__ void k_grid_ic(int Ni, double rratio, double* r) {
  int n = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (n > Ni) return;
  const double PI = 3.1415926535897931;
  const int N_ = 2 * Ni, np = n + Ni;
  const double ri = rratio / (1.0 - rratio);
  const double x = ri * cos(PI * (N_ - np) / (double)(N_ - 1));
  for (int p = -3; p <= 3; ++p) {
    double y = 1.0;
    int ap = p < 0 ? -p : p;
    for (int k = 0; k < ap; ++k) y = (k == 0) ? x : y * x;
    r[(size_t)(p + 3) * Ni + (n - 1)] = p < 0 ? 1.0 / y : (p == 1 ? x : y);
  }
}

// leg_gwP0 (legendre.F90:103-104): P_0^0 * gw / 2 on both hemispheres
__global__ void k_gwP0(int Th, int Th2, const double* leg_P, const double* gw, double* gwP0) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Th2) return;
  const double v = leg_P[j] * gw[j] * 0.5;  // table P, harmonic nh = 0 (l = m = 0)
  gwP0[j] = v;
  gwP0[Th - 1 - j] = v;
}

// FD weights at point n by inverting the local Taylor matrix; integration-weight
// contributions w(n, i, j) kept for an ordered sum.
__global__ void k_fdweights(int N, int KL, const double* r, double* dr, double* wcontrib, int* fail) {
  int n = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (n > N) return;
  const int lda = 2 * KL + 1;
  double A[(2 * LSD_MAX_KL + 1) * (2 * LSD_MAX_KL + 1)];
  const double* r1 = r + (size_t)4 * N;  // r^1
  const double* r2 = r + (size_t)5 * N;  // r^2
#define Aa(i, j) A[((i) - 1) + lda * ((j) - 1)]
  int l = max(1, n - KL), rr = min(n + KL, N), nn = rr - l + 1;
  for (int i = 1; i <= nn; ++i) Aa(i, 1) = 1.0;
  for (int j = 2; j <= nn; ++j)
    for (int i = 1; i <= nn; ++i) Aa(i, j) = Aa(i, j - 1) * (r1[l + i - 2] - r1[n - 1]) / (double)(j - 1);
  if (dev_mat_invert(nn, A, lda) != 0) { atomicExch(fail, 3); return; }
  const size_t band = (size_t)(2 * KL + 1) * N;
  for (int i = 1; i <= KL; ++i)
    for (int j = l; j <= rr; ++j) dr[(i - 1) * band + (size_t)(KL + n - j) + (size_t)(2 * KL + 1) * (j - 1)] = Aa(i + 1, j - l + 1);
  double c = 1.0, e = 1.0;
  for (int i = 1; i <= nn; ++i) {
    c = c * (r1[min(n + 1, N) - 1] - r1[n - 1]) / (double)i;
    e = e * (r1[max(1, n - 1) - 1] - r1[n - 1]) / (double)i;
    for (int j = l; j <= rr; ++j) {
      double w = 0.5 * (c - e) * Aa(i, j - l + 1) * r2[n - 1];
      wcontrib[((size_t)(n - 1) * lda + (i - 1)) * lda + (j - l)] = w;
    }
  }
#undef Aa
}

// intr2dr(j) = sum over n ascending, i ascending of the contributions (meshs.F90:311-336),
// with the weighted variants wts[4][N]: intr2dr_comp (rho), intr2dr_compS (rho T),
// intr2dr_magdiss (eta), intr2dr_veldiss (2 rho (dxi/dr - xi^2/3))
__global__ void k_intr2dr(int N, int KL, const double* wcontrib, const double* ref, double* intr2dr, double* wts) {
  int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (j > N) return;
  const int lda = 2 * KL + 1;
  double s = 0.0, sc = 0.0, ss = 0.0, sm = 0.0, sv = 0.0;
  for (int n = max(1, j - KL); n <= min(j + KL, N); ++n) {
    int l = max(1, n - KL), rr = min(n + KL, N), nn = rr - l + 1;
    const double rho = ref[n - 1], xi = ref[N + n - 1], dxi = ref[2 * N + n - 1];
    const double T = ref[3 * N + n - 1], eta = ref[5 * N + n - 1];
    for (int i = 1; i <= nn; ++i) {
      const double w = wcontrib[((size_t)(n - 1) * lda + (i - 1)) * lda + (j - l)];
      s = s + w;
      sc = sc + w * rho;
      ss = ss + w * (rho * T);
      sm = sm + w * eta;
      sv = sv + w * 2.0 * rho * (dxi - xi * xi / 3.0);
    }
  }
  intr2dr[j - 1] = s;
  wts[j - 1] = sc;
  wts[N + j - 1] = ss;
  wts[2 * N + j - 1] = sm;
  wts[3 * N + j - 1] = sv;
}

// radLap = dr2 + dr1*2/r ; r1dr = dr1 + diag(1/r) ; the reference-state bands
// laps[LAP_*] and compr1dr = dr1 + diag(1/r + xi)   (meshs.F90:339-415)
__global__ void k_bands(int N, int KL, const double* r, const double* dr, const double* ref, double* radlap,
                        double* r1dr, double* laps, double* compr1dr) {
  int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (j > N) return;
  const size_t band = (size_t)(2 * KL + 1) * N;
  const double* rm1 = r + (size_t)2 * N;
  const double* xi = ref + N;
  const double* eta = ref + (size_t)5 * N;
  const double* deta = ref + (size_t)6 * N;
  for (int row = 1; row <= 2 * KL + 1; ++row) {
    size_t id = (size_t)(row - 1) + (size_t)(2 * KL + 1) * (j - 1);
    int n = row - KL - 1 + j;
    double v = 0.0, cl = 0.0, gl = 0.0, mt = 0.0, mp = 0.0;
    if (n >= 1 && n <= N) {
      const double d1 = dr[id], d2 = dr[band + id];
      v = d2 + d1 * 2.0 * rm1[n - 1];
      cl = d2 + 2.0 * (xi[n - 1] + rm1[n - 1]) * d1;                          // CompLap
      mt = eta[n - 1] * (d2 + 2.0 * rm1[n - 1] * d1) + deta[n - 1] * d1;     // MagTorLap
      mp = eta[n - 1] * (d2 + 2.0 * rm1[n - 1] * d1);                        // MagPolLap
      gl = d2 + (xi[n - 1] + 2.0 * rm1[n - 1]) * d1;                          // GreLap
    }
    radlap[id] = v;
    laps[LAP_COMP * band + id] = cl;
    laps[LAP_GRE * band + id] = gl;
    laps[LAP_MAGTOR * band + id] = mt;
    laps[LAP_MAGPOL * band + id] = mp;
    double w = dr[id];
    if (row == KL + 1) w = w + rm1[j - 1];
    r1dr[id] = w;
    double wc = dr[id];
    if (row == KL + 1) wc = wc + rm1[j - 1] + xi[j - 1];
    compr1dr[id] = wc;
  }
}

// ---------------------------------------------------------------------------------------
// Operators.  One thread per (family, l): build X in LAPACK band storage, apply the
// boundary rows, factorise; build Y in the solve layout [fam][N][2KL+1][L].
// ---------------------------------------------------------------------------------------
struct OpParams {
  double c1[OP_NFAM], c2_[OP_NFAM], c2y[OP_NFAM];  // X = c1 / dt + c2_ (.), Y = c1 / dt - c2y (.)
  double Hyp;
  int vel_bc, cod_bc, comp_bc;
  int anelastic;
};

// The diagonal term d of an anelastic operator family at shell n (1-based); X gets
// c1_ + c2_ d and Y gets c1_ - c2y d on the diagonal (timestep.F90:47-128, 214-546).
__device__ double anel_diag(int fam, int l, int n, int N, const double* r, const double* ref, double Hyp) {
  const double ll1 = (double)(l * (l + 1));
  const double rm1 = r[(size_t)2 * N + n - 1], rm2 = r[(size_t)1 * N + n - 1];
  const double xi = ref[N + n - 1], dxi = ref[2 * N + n - 1];
  const double eta = ref[5 * N + n - 1], deta = ref[6 * N + n - 1];
  const double t = ll1 * rm2;
  double d;
  switch (fam) {
    case OP_VTOR:
    case OP_VPOL:  // tim_lumesh_vel_X / tim_mesh_vel_Y
      d = t + Hyp * (t * t);
      d = d - 2.0 * xi * rm1;
      d = d - xi * xi;
      return d - dxi;
    case OP_VGRE:  // tim_lumesh_Gre_X
      d = t - xi * rm1;
      return d - dxi;
    case OP_MTOR:  // tim_iclumesh_Tor_X / tim_mesh_mag_Tor_Y
      d = ll1 * eta * rm2;
      d = d - deta * rm1;
      return d + Hyp * (t * t);
    case OP_MPOL:  // tim_iclumesh_Pol_X / tim_mesh_mag_Pol_Y
      d = ll1 * eta * rm2;
      return d + Hyp * (t * t);
    default:  // tim_lumesh_X / tim_mesh_Y (codensity, composition)
      return t + Hyp * (t * t);
  }
}

// One warp per (family, l): the lanes build the band in shared memory, lane 0 factorises
// it there (dgbtf2 at shared-memory latency: one matrix per thread on global memory took
// 1.3 ms per rebuild at L = 128, N = 129), and the lanes write it out.  wpb warps per CTA.
__global__ void k_build_ops(int N, int NL, int KL, int L, int wpb, const double* r, const double* dr,
                            const double* radlap, const double* laps, const double* ref, OpParams P,
                            const double* dtp, double* lu, int* ipiv, double* y, int* info) {
  extern __shared__ double osm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int l = blockIdx.x * wpb + warp;
  const int fam = blockIdx.y;
  if (l >= L) return;
  const int ld = 3 * KL + 1, ldm = 2 * KL + 1;
  double* A = osm + (size_t)warp * ld * N;
  double* Ag = lu + ((size_t)fam * L + l) * (size_t)ld * NL;  // NL: the families' row stride
  int* ip = ipiv + ((size_t)fam * L + l) * NL;
  const double* rm1 = r + (size_t)2 * N;
  const double* rm2 = r + (size_t)1 * N;
  const size_t band = (size_t)ldm * N;
#define AX(i, j) A[(size_t)((i) - 1) + (size_t)ld * ((j) - 1)]
#define MB(B, i, j) (B)[(size_t)((i) - 1) + (size_t)ldm * ((j) - 1)]
  for (int i = lane; i < ld * N; i += 32) A[i] = 0.0;
  __syncwarp();
  bool skip_l0 = (fam != OP_COD && fam != OP_COMP);
  if (l == 0 && skip_l0) {  // never solved: keep an identity so the factors are defined
    for (int j = 1 + lane; j <= N; j += 32) AX(2 * KL + 1, j) = 1.0;
    __syncwarp();
    if (lane == 0) info[fam * L + l] = dev_dgbtf2(N, KL, A, ld, ip);
    __syncwarp();
    for (int i = lane; i < ld * N; i += 32) Ag[i] = A[i];
    return;
  }
  const double c1_ = P.c1[fam] / *dtp, c2_ = P.c2_[fam], c2y = P.c2y[fam];  // c1 / dt
  const double ll1 = (double)(l * (l + 1));
  // A(KL+1:, :) = -c2_ * Lap.  Boussinesq: radLap == radLap_flayer == GreLap == MagTorLap
  // == MagPolLap bit for bit (f_factor = 1, xi = 0, eta = 1, deta = 0); anelastic: CompLap
  // (velocity), GreLap (Green's, codensity, composition), MagTorLap, MagPolLap.
  const double* lap = radlap;
  if (P.anelastic) {
    const int which = (fam == OP_VTOR || fam == OP_VPOL) ? LAP_COMP
                    : fam == OP_MTOR ? LAP_MAGTOR : fam == OP_MPOL ? LAP_MAGPOL : LAP_GRE;
    lap = laps + which * band;
  }
  for (int j = 1 + lane; j <= N; j += 32)
    for (int row = 1; row <= ldm; ++row) {
      double v = MB(lap, row, j);
      AX(KL + row, j) = (fam == OP_MTOR || fam == OP_MPOL) ? 0.0 - c2_ * v : -c2_ * v;
    }
  __syncwarp();
  for (int n = 1 + lane; n <= N; n += 32) {
    double t = ll1 * rm2[n - 1];
    if (P.anelastic)
      AX(2 * KL + 1, n) = AX(2 * KL + 1, n) + c1_ + c2_ * anel_diag(fam, l, n, N, r, ref, P.Hyp);
    else if (fam == OP_MTOR || fam == OP_MPOL)
      AX(2 * KL + 1, n) = AX(2 * KL + 1, n) + c1_ + c2_ * ll1 * rm2[n - 1];
    else
      AX(2 * KL + 1, n) = AX(2 * KL + 1, n) + c1_ + c2_ * (t + P.Hyp * t * t);
  }
  __syncwarp();
  if (lane == 0) {  // boundary rows, then the factorisation
    for (int j = 1; j <= 1 + KL; ++j) AX(2 * KL + 1 + 1 - j, j) = 0.0;
    for (int j = N - KL; j <= N; ++j) AX(2 * KL + 1 + N - j, j) = 0.0;
    switch (fam) {
      case OP_VTOR:  // vel_bc_Tor (velocity.F90:177-201)
        if (P.vel_bc == 1 || P.vel_bc == 2) AX(2 * KL + 1, 1) = 1.0;
        else {
          for (int j = 1; j <= 1 + KL; ++j) AX(2 * KL + 1 + 1 - j, j) = MB(dr, KL + 1 + 1 - j, j);
          AX(2 * KL + 1, 1) = AX(2 * KL + 1, 1) - rm1[0];
        }
        if (P.vel_bc == 1 || P.vel_bc == 3) AX(2 * KL + 1, N) = 1.0;
        else {
          for (int j = N - KL; j <= N; ++j) AX(2 * KL + 1 + N - j, j) = MB(dr, KL + 1 + N - j, j);
          AX(2 * KL + 1, N) = AX(2 * KL + 1, N) - rm1[N - 1];
        }
        break;
      case OP_VPOL: {  // vel_bc_Pol (velocity.F90:207-254); anelastic stress-free adds xi dr
        const double xi1 = P.anelastic ? ref[N] : 0.0, xiN = P.anelastic ? ref[2 * N - 1] : 0.0;
        if (P.vel_bc == 1 || P.vel_bc == 2)
          for (int j = 1; j <= 1 + KL; ++j) AX(2 * KL + 1 + 1 - j, j) = MB(dr, KL + 1 + 1 - j, j);
        else if (!P.anelastic)
          for (int j = 1; j <= 1 + KL; ++j) AX(2 * KL + 1 + 1 - j, j) = MB(dr + band, KL + 1 + 1 - j, j);
        else
          for (int j = 1; j <= 1 + KL; ++j)
            AX(2 * KL + 1 + 1 - j, j) = MB(dr + band, KL + 1 + 1 - j, j) + xi1 * MB(dr, KL + 1 + 1 - j, j);
        if (P.vel_bc == 1 || P.vel_bc == 3)
          for (int j = N - KL; j <= N; ++j) AX(2 * KL + 1 + N - j, j) = MB(dr, KL + 1 + N - j, j);
        else if (!P.anelastic)
          for (int j = N - KL; j <= N; ++j) AX(2 * KL + 1 + N - j, j) = MB(dr + band, KL + 1 + N - j, j);
        else
          for (int j = N - KL; j <= N; ++j)
            AX(2 * KL + 1 + N - j, j) = MB(dr + band, KL + 1 + N - j, j) + xiN * MB(dr, KL + 1 + N - j, j);
        break;
      }
      case OP_VGRE:  // vel_bc_Gre (velocity.F90:260-267)
        AX(2 * KL + 1, 1) = 1.0;
        AX(2 * KL + 1, N) = 1.0;
        break;
      case OP_COD:
      case OP_COMP: {  // cod_bc_C (codensity.F90:85-112)
        int bc = fam == OP_COD ? P.cod_bc : P.comp_bc;
        if (bc == 1 || bc == 2) AX(2 * KL + 1, 1) = 1.0;
        else for (int j = 1; j <= 1 + KL; ++j) AX(2 * KL + 1 + 1 - j, j) = MB(dr, KL + 1 + 1 - j, j);
        if (bc == 1 || bc == 3) AX(2 * KL + 1, N) = 1.0;
        else for (int j = N - KL; j <= N; ++j) AX(2 * KL + 1 + N - j, j) = MB(dr, KL + 1 + N - j, j);
        break;
      }
      case OP_MTOR:  // mag_bc_Tor (magnetic.F90:137-192), Ni = 1
        AX(2 * KL + 1, 1) = 1.0;
        AX(2 * KL + 1, N) = 1.0;
        break;
      case OP_MPOL:  // mag_bc_Pol (magnetic.F90:198-282), insulating, Ni = 1
        for (int j = 1; j <= 1 + KL; ++j) AX(2 * KL + 1 + 1 - j, j) = MB(dr, KL + 1 + 1 - j, j);
        AX(2 * KL + 1, 1) = AX(2 * KL + 1, 1) - rm1[0] * l;
        for (int j = N - KL; j <= N; ++j) AX(2 * KL + 1 + N - j, j) = MB(dr, KL + 1 + N - j, j);
        AX(2 * KL + 1, N) = AX(2 * KL + 1, N) + rm1[N - 1] * (l + 1);
        break;
    }
    info[fam * L + l] = dev_dgbtf2(N, KL, A, ld, ip);
  }
  __syncwarp();
  for (int i = lane; i < ld * N; i += 32) Ag[i] = A[i];
  // Y = c2y*Lap ; diag += c1_ - c2y*(l(l+1)/r^2 + Hyp (.)^2)   (tim_mesh_Y / _flayer_Y;
  // anelastic: tim_mesh_vel_Y, tim_mesh_Y, tim_mesh_mag_Tor_Y / _Pol_Y)
  if (fam != OP_VGRE) {
    for (int j = 1 + lane; j <= N; j += 32)
      for (int row = 1; row <= ldm; ++row) {
        double v = c2y * MB(lap, row, j);
        if (row == KL + 1) {
          double t = (double)(l * (l + 1)) * rm2[j - 1];
          if (P.anelastic) v = v + c1_ - c2y * anel_diag(fam, l, j, N, r, ref, P.Hyp);
          else v = v + c1_ - c2y * (t + P.Hyp * t * t);
        }
        y[(((size_t)fam * L + l) * N + (j - 1)) * ldm + (row - 1)] = v;
      }
  }
#undef AX
#undef MB
}

// LAPACK layouts [fam][L][N][band] -> solve layouts [fam][N][band][L] (degree fastest),
// for the factors, the pivots and the Y bands
// (factors and pivots with the row stride NL; the field families of a conducting inner
// core have NL rows, the others N)
__global__ void k_lu_transpose(int N, int NL, int icfam, int KL, int L, const double* lu, const int* ipiv,
                               const double* y, double* lus, int* ipivs, double* yt) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  int fam = blockIdx.z;
  if (l >= L) return;
  const bool coupled = icfam && (fam == OP_MTOR || fam == OP_MPOL);
  if (j >= (coupled ? NL : N)) return;
  const int ld = 3 * KL + 1, ldm = 2 * KL + 1;
  const double* A = lu + (((size_t)fam * L + l) * NL + j) * ld;
  for (int row = 0; row < ld; ++row) lus[(((size_t)fam * NL + j) * ld + row) * L + l] = A[row];
  ipivs[((size_t)fam * NL + j) * L + l] = ipiv[((size_t)fam * L + l) * NL + j];
  if (j >= N) return;
  const double* Y = y + (((size_t)fam * L + l) * N + j) * ldm;
  for (int row = 0; row < ldm; ++row) yt[(((size_t)fam * N + j) * ldm + row) * L + l] = Y[row];
}

// The field's operators with a conducting inner core, Boussinesq (tim_iclumesh_Tor_X /
// _Pol_X, timestep.F90:218-344; mag_bc_Tor / mag_bc_Pol, magnetic.F90:137-282): NL = Ni +
// N - 1 unknowns, 1..Ni on the inner core's mesh and Ni..NL on the outer core's (Ni the
// inner-core boundary, shared); row 1 the innermost point's condition, row Ni the
// continuity of dr across the boundary, row NL the insulating exterior.  Also the inner
// core's Y bands (tim_mesh_Y on its mesh) in the solve layout [k][Ni][2KL+1][L].
// One warp per (l, k), k = 0 toroidal, 1 poloidal, in shared memory as k_build_ops.
__global__ void k_build_icops(int N, int Ni, int KL, int L, int wpb, const double* r, const double* dr,
                              const double* radlap, const double* icr, const double* icdr, const double* icradlap,
                              OpParams P, const double* dtp, double* lu, int* ipiv, double* icyt, int* info) {
  extern __shared__ double osm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int l = blockIdx.x * wpb + warp, k = blockIdx.y;
  if (l >= L) return;
  const int fam = k == 0 ? OP_MTOR : OP_MPOL;
  const int NL = N + Ni - 1, ld = 3 * KL + 1, ldm = 2 * KL + 1;
  double* A = osm + (size_t)warp * ld * NL;
  double* Ag = lu + ((size_t)fam * L + l) * (size_t)ld * NL;
  int* ip = ipiv + ((size_t)fam * L + l) * NL;
#define AX(i, j) A[(size_t)((i) - 1) + (size_t)ld * ((j) - 1)]
#define MB(B, i, j) (B)[(size_t)((i) - 1) + (size_t)ldm * ((j) - 1)]
  for (int i = lane; i < ld * NL; i += 32) A[i] = 0.0;
  __syncwarp();
  if (l == 0) {  // never solved
    for (int j = 1 + lane; j <= NL; j += 32) AX(2 * KL + 1, j) = 1.0;
    __syncwarp();
    if (lane == 0) info[fam * L + l] = dev_dgbtf2(NL, KL, A, ld, ip);
    __syncwarp();
    for (int i = lane; i < ld * NL; i += 32) Ag[i] = A[i];
    return;
  }
  const double c1_ = P.c1[fam] / *dtp, c2_ = P.c2_[fam], c2y = P.c2y[fam];  // c1 / dt
  const double ll1 = (double)(l * (l + 1));
  const double* rm2 = r + (size_t)1 * N;
  const double* rm1 = r + (size_t)2 * N;
  const double* icrm2 = icr + (size_t)1 * Ni;
  const double* icrm1 = icr + (size_t)2 * Ni;
  const size_t icband = (size_t)ldm * Ni;
  // the phases keep the reference's order of additions on the shared column Ni; lanes
  // split the columns within a phase
  for (int j = 1 + lane; j <= Ni; j += 32)
    for (int row = 1; row <= ldm; ++row) AX(KL + row, j) = -c2_ * MB(icradlap, row, j);
  __syncwarp();
  for (int n = 1 + lane; n <= Ni; n += 32) AX(2 * KL + 1, n) = AX(2 * KL + 1, n) + c1_ + c2_ * ll1 * icrm2[n - 1];
  __syncwarp();
  for (int j = 1 + lane; j <= N; j += 32)
    for (int row = 1; row <= ldm; ++row) AX(KL + row, j + Ni - 1) = AX(KL + row, j + Ni - 1) - c2_ * MB(radlap, row, j);
  __syncwarp();
  for (int n = 1 + lane; n <= N; n += 32) AX(2 * KL + 1, n + Ni - 1) = AX(2 * KL + 1, n + Ni - 1) + c1_ + c2_ * ll1 * rm2[n - 1];
  __syncwarp();
  if (lane == 0) {  // boundary rows, then the factorisation
    for (int j = 1; j <= 1 + KL; ++j) AX(2 * KL + 1 + 1 - j, j) = 0.0;
    for (int j = NL - KL; j <= NL; ++j) AX(2 * KL + 1 + NL - j, j) = 0.0;
    for (int j = Ni - KL; j <= Ni + KL; ++j) AX(2 * KL + 1 + Ni - j, j) = 0.0;
    if (k == 0) {  // BTor = 0 at the innermost point and outside
      AX(2 * KL + 1, 1) = 1.0;
      AX(2 * KL + 1, NL) = 1.0;
    } else {  // (dr - l/r) BPol = 0 innermost, (dr + (l+1)/r) BPol = 0 at the outer wall
      for (int j = 1; j <= 1 + KL; ++j) AX(2 * KL + 1 + 1 - j, j) = MB(icdr, KL + 1 + 1 - j, j);
      AX(2 * KL + 1, 1) = AX(2 * KL + 1, 1) - icrm1[0] * l;
      for (int j = N - KL; j <= N; ++j) {
        const int j_ = j + Ni - 1;
        AX(2 * KL + 1 + NL - j_, j_) = MB(dr, KL + 1 + N - j, j);
      }
      AX(2 * KL + 1, NL) = AX(2 * KL + 1, NL) + rm1[N - 1] * (l + 1);
    }
    for (int j = 2; j <= 1 + KL; ++j) {  // dr continuous across the inner-core boundary
      const int j_ = j + Ni - 1;
      AX(2 * KL + 1 + Ni - j_, j_) = MB(dr, KL + 1 + 1 - j, j);
    }
    for (int j = Ni - KL; j <= Ni - 1; ++j) AX(2 * KL + 1 + Ni - j, j) = -MB(icdr, KL + 1 + Ni - j, j);
    AX(2 * KL + 1, Ni) = MB(dr, KL + 1, 1) - MB(icdr, KL + 1, Ni);
    info[fam * L + l] = dev_dgbtf2(NL, KL, A, ld, ip);
  }
  __syncwarp();
  for (int i = lane; i < ld * NL; i += 32) Ag[i] = A[i];
  for (int j = 1 + lane; j <= Ni; j += 32)  // tim_mesh_Y on the inner core's mesh
    for (int row = 1; row <= ldm; ++row) {
      double v = c2y * MB(icradlap, row, j);
      if (row == KL + 1) {
        const double t = ll1 * icrm2[j - 1];
        v = v + c1_ - c2y * (t + P.Hyp * t * t);
      }
      icyt[(((size_t)k * Ni + (j - 1)) * ldm + (row - 1)) * L + l] = v;
    }
  (void)icband;
#undef AX
#undef MB
}

}  // namespace

// ---------------------------------------------------------------------------------------
int lsd_build_tables(lsd_ctx* ctx) {
  const int Th = ctx->Th, Th2 = ctx->Th2, H = ctx->H, N = ctx->N, KL = ctx->KL, L = ctx->L, M = ctx->M;
  cudaStream_t s = ctx->stream;
  int* d_fail = nullptr;
  CUDA_TRY(cudaMalloc(&d_fail, sizeof(int)));
  CUDA_TRY(cudaMemsetAsync(d_fail, 0, sizeof(int), s));
  k_gauss<<<ceil_div((Th + 1) / 2, 128), 128, 0, s>>>(Th, ctx->d_gp, ctx->d_gw, d_fail);
  k_trig<<<ceil_div(Th, 128), 128, 0, s>>>(Th, ctx->d_gp, ctx->d_sn, ctx->d_sn1);
  dim3 gl(ceil_div(Th2, 64), M);
  k_legendre<<<gl, 64, 0, s>>>(L, M, ctx->Mp, H, Th2, ctx->d_gp, ctx->d_gw, ctx->d_sn1, ctx->d_lm2nh, ctx->d_leg, d_fail);
  k_gwP0<<<ceil_div(Th2, 128), 128, 0, s>>>(Th, Th2, ctx->d_leg, ctx->d_gw, ctx->d_gwP0);
  ctx->launches += 4;
  CUDA_TRY(cudaGetLastError());
  int fail = 0;
  CUDA_TRY(cudaMemcpyAsync(&fail, d_fail, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  cudaFree(d_fail);
  if (fail == 2) return lsd_fail(ctx, LSD_EARG, "schnla: sin(theta) too small (legendre)");
  if (fail) return lsd_fail(ctx, LSD_ESINGULAR, "table construction failed (code " + std::to_string(fail) + ")");
  return lsd_build_radial(ctx);
}

// mes_precompute / mes_rdom_init (meshs.F90:116-419) on the current reference state
int lsd_build_radial(lsd_ctx* ctx) {
  const int N = ctx->N, KL = ctx->KL;
  cudaStream_t s = ctx->stream;
  int* d_fail = nullptr;
  CUDA_TRY(cudaMalloc(&d_fail, sizeof(int)));
  CUDA_TRY(cudaMemsetAsync(d_fail, 0, sizeof(int), s));
  k_grid<<<ceil_div(N, 128), 128, 0, s>>>(N, ctx->cfg.rratio, ctx->cfg.alpha, ctx->d_r);
  double* wc = nullptr;
  size_t lda = 2 * KL + 1;
  CUDA_TRY(cudaMalloc(&wc, sizeof(double) * N * lda * lda));
  CUDA_TRY(cudaMemsetAsync(ctx->d_dr, 0, sizeof(double) * KL * lda * N, s));
  k_fdweights<<<ceil_div(N, 64), 64, 0, s>>>(N, KL, ctx->d_r, ctx->d_dr, wc, d_fail);
  k_intr2dr<<<ceil_div(N, 128), 128, 0, s>>>(N, KL, wc, ctx->d_ref, ctx->d_intr2dr, ctx->d_wts);
  k_bands<<<ceil_div(N, 128), 128, 0, s>>>(N, KL, ctx->d_r, ctx->d_dr, ctx->d_ref, ctx->d_radlap, ctx->d_r1dr,
                                           ctx->d_laps, ctx->d_compr1dr);
  ctx->launches += 4;
  double* wci = nullptr;
  if (ctx->Nic > 1) {  // the inner core's mesh: the same construction on its Nic points
    const int Ni = ctx->Nic;
    CUDA_TRY(cudaMalloc(&wci, sizeof(double) * Ni * lda * lda));
    CUDA_TRY(cudaMemsetAsync(ctx->d_icdr, 0, sizeof(double) * KL * lda * Ni, s));
    k_grid_ic<<<ceil_div(Ni, 128), 128, 0, s>>>(Ni, ctx->cfg.rratio, ctx->d_icr);
    k_fdweights<<<ceil_div(Ni, 64), 64, 0, s>>>(Ni, KL, ctx->d_icr, ctx->d_icdr, wci, d_fail);
    k_intr2dr<<<ceil_div(Ni, 128), 128, 0, s>>>(Ni, KL, wci, ctx->d_icref, ctx->d_icintr2dr, ctx->d_icwts);
    k_bands<<<ceil_div(Ni, 128), 128, 0, s>>>(Ni, KL, ctx->d_icr, ctx->d_icdr, ctx->d_icref, ctx->d_icradlap,
                                              ctx->d_icr1dr, ctx->d_iclaps, ctx->d_iccompr1dr);
    ctx->launches += 4;
  }
  CUDA_TRY(cudaGetLastError());
  int fail = 0;
  CUDA_TRY(cudaMemcpyAsync(&fail, d_fail, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  cudaFree(wc);
  if (wci) cudaFree(wci);
  cudaFree(d_fail);
  if (fail) return lsd_fail(ctx, LSD_ESINGULAR, "radial mesh construction failed (code " + std::to_string(fail) + ")");
  return LSD_OK;
}

namespace {
// After an operator build: the step's dt into rot's slot (rot_predictor / rot_corrector
// read it there), and LSD_ESINGULAR into *status (when given) if a factorisation met a
// zero pivot (mes_lu_find, meshs.F90:447-473) or an influence matrix was singular.
__global__ void k_ops_finish(const double* dtp, double* rot_dt, const int* info, int ninfo, const int* fail,
                             int* status) {
  __shared__ int bad;
  if (threadIdx.x == 0) { bad = *fail; *rot_dt = *dtp; }
  __syncthreads();
  for (int i = threadIdx.x; i < ninfo; i += blockDim.x)
    if (info[i] != 0) bad = 1;
  __syncthreads();
  if (threadIdx.x == 0 && bad && status && *status == LSD_OK) *status = LSD_ESINGULAR;
}
}  // namespace

// vel_matrices + cod_matrices + comp_matrices + mag_matrices (velocity.F90:56-168,
// codensity.F90:37-79, magnetic.F90:62-133) at the dt held in device memory (*dtp): only
// launches and memsets on the context's stream, no allocation and no host
// synchronisation, so the one-graph step captures it (run when tim_new_tstep changes dt).
int lsd_launch_operator_build(lsd_ctx* ctx, const double* dtp, int* status) {
  const int N = ctx->N, KL = ctx->KL, L = ctx->L;
  const lsd_config& c = ctx->cfg;
  cudaStream_t s = ctx->stream;
  OpParams P;
  const double impl = c.implicit;
  auto setf = [&](int fam, double c1, double c2) {
    P.c1[fam] = c1;
    P.c2_[fam] = (impl == 0.0) ? 1.0 : c2 * impl;
    P.c2y[fam] = c2 * (1.0 - impl);
  };
  setf(OP_VTOR, 1.0, c.Pm);
  setf(OP_VPOL, 1.0, c.Pm);
  setf(OP_VGRE, 0.0, 1.0 / impl);
  setf(OP_COD, c.Pr / c.Pm, 1.0);
  setf(OP_COMP, c.Sc / c.Pm, 1.0);
  setf(OP_MTOR, 1.0, 1.0);
  setf(OP_MPOL, 1.0, 1.0);
  P.Hyp = c.Hyp;
  P.vel_bc = c.vel_bc; P.cod_bc = c.cod_bc; P.comp_bc = c.comp_bc;
  P.anelastic = c.boussinesq ? 0 : 1;
  CUDA_TRY(cudaMemsetAsync(ctx->d_opfail, 0, sizeof(int), s));
  CUDA_TRY(cudaMemsetAsync(ctx->d_y, 0, sizeof(double) * OP_NFAM * N * (2 * KL + 1) * L, s));
  const int NL = ctx->NL, Ni = ctx->Nic;
  // one warp per operator, its band in shared memory: up to four per CTA within 200 KB
  auto warps_for = [&](int cols) {
    const size_t per = sizeof(double) * (size_t)(3 * KL + 1) * cols;
    return (int)std::min<size_t>(4, (size_t)(200 * 1024) / per);
  };
  const int wpb = warps_for(N), wpbi = warps_for(NL);
  if (wpb < 1 || wpbi < 1)
    return lsd_fail(ctx, LSD_EARG, "operator build: the band of one operator exceeds 200 KB of shared memory");
  const size_t smem = sizeof(double) * (size_t)(3 * KL + 1) * N * wpb;
  const size_t smemi = sizeof(double) * (size_t)(3 * KL + 1) * NL * wpbi;
  CUDA_TRY(cudaFuncSetAttribute(k_build_ops, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 g(ceil_div(L, wpb), OP_NFAM);
  k_build_ops<<<g, 32 * wpb, smem, s>>>(N, NL, KL, L, wpb, ctx->d_r, ctx->d_dr, ctx->d_radlap, ctx->d_laps,
                                        ctx->d_ref, P, dtp, ctx->d_lu, ctx->d_ipiv, ctx->d_y, ctx->d_info);
  if (Ni > 1) {  // the field families coupled to the inner core
    CUDA_TRY(cudaFuncSetAttribute(k_build_icops, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemi));
    k_build_icops<<<dim3(ceil_div(L, wpbi), 2), 32 * wpbi, smemi, s>>>(
        N, Ni, KL, L, wpbi, ctx->d_r, ctx->d_dr, ctx->d_radlap, ctx->d_icr, ctx->d_icdr, ctx->d_icradlap, P, dtp,
        ctx->d_lu, ctx->d_ipiv, ctx->d_icyt, ctx->d_info);
    ctx->launches++;
  }
  dim3 gt(ceil_div(L, 64), NL, OP_NFAM);
  k_lu_transpose<<<gt, 64, 0, s>>>(N, NL, Ni > 1 ? 1 : 0, KL, L, ctx->d_lu, ctx->d_ipiv, ctx->d_y, ctx->d_lus,
                                   ctx->d_ipivs, ctx->d_yt);
  CUDA_TRY(cudaMemsetAsync(ctx->d_gret, 0, sizeof(double) * 2 * N * L, s));
  {
    int rc = lsd_launch_greens(ctx, ctx->d_opfail);  // on the solve-layout factors
    if (rc) return rc;
  }
  k_ops_finish<<<1, 256, 0, s>>>(dtp, ctx->d_rot + ROT_DT, ctx->d_info, OP_NFAM * L, ctx->d_opfail, status);
  ctx->launches += 3;
  CUDA_TRY(cudaGetLastError());
  return LSD_OK;
}

// The operators at the host's dt (lsd_create, lsd_set_time, the host-controlled step):
// dt to the device control block, the build, then the checks with their messages.
int lsd_build_operators(lsd_ctx* ctx) {
  const int L = ctx->L;
  cudaStream_t s = ctx->stream;
  const double dt = ctx->dt;
  ctx->h_red[LSD_HRED_DT] = dt;
  CUDA_TRY(cudaMemcpyAsync(&ctx->d_pc->s.dt, ctx->h_red + LSD_HRED_DT, sizeof(double), cudaMemcpyHostToDevice, s));
  int rc = lsd_launch_operator_build(ctx, &ctx->d_pc->s.dt, nullptr);
  if (rc) return rc;
  std::vector<int> info((size_t)OP_NFAM * L);
  int fail = 0;
  CUDA_TRY(cudaMemcpyAsync(info.data(), ctx->d_info, sizeof(int) * info.size(), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(&fail, ctx->d_opfail, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  for (int fam = 0; fam < OP_NFAM; ++fam)
    for (int l = 0; l < L; ++l)
      if (info[(size_t)fam * L + l] != 0)
        return lsd_fail(ctx, LSD_ESINGULAR, "mes_lu_find: zero pivot in operator family " + std::to_string(fam) +
                                                " l=" + std::to_string(l));
  if (fail) return lsd_fail(ctx, LSD_ESINGULAR, "influence matrix inversion failed (vel_matrices)");
  ctx->have_ops = true;
  ctx->op_dt = dt;
  return LSD_OK;
}
