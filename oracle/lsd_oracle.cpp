// lsd_oracle.cpp -- CPU FP64 restatement of the Leeds dynamo timestep hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU baseline:
// only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may
// load it.  The product (leeds-code_b200/) never links, imports or calls it.
//
// It restates, loop for loop, the Fortran reference Leeds-Spherical-Dynamo/leeds-code
// v3.6.0 (paths below are relative to that project):
//   auxiliary/gauwts.f, schnla.f, pmm.f, pmm1.f, plm.f, dpmm.f, dpmm1.f, dplm.f
//   modules/legendre.F90, meshs.F90, variables.F90, transform.fftw3.F90 (serial
//   branches), nonlinear.F90, timestep.F90, velocity.F90, codensity.F90,
//   composition.F90, magnetic.F90; program/main.F90 (main loop); program/io.F90
//   (energy diagnostics, state-file harmonic order).
// Two third-party dependencies of the reference are restated from their published
// contracts, since neither is vendored in the reference tree:
//   * FFTW3 (version unpinned; the Makefile comments name fftw/3.3.8): the unnormalised
//     DFT of dfftw_plan_many_dft_c2r / _r2c (FFTW manual 4.8), restated here as a
//     mixed-radix complex FFT.  The c2r ignores the imaginary parts of the DC and
//     Nyquist bins; the r2c returns exact zero imaginary parts there.
//   * LAPACK (version unpinned): dgbtrf/dgbtf2 and dgbtrs/dtbsv (banded LU with
//     partial pivoting and its solve), dgetrf/dgetf2 + dgetri/dtrtri (small inverses),
//     restated from the reference LAPACK algorithms.  tests/ pin these against scipy's
//     LAPACK (scipy.linalg.lapack.dgbtrf/dgbtrs).
// Scope: Boussinesq or anelastic MHD + codensity (+ composition) with an insulating
// inner core (i_Nic = 1), or Boussinesq with a conducting inner core (i_Nic > 1, no-slip
// inner wall) and its rotation (b_rot_tstep), fixed dt (d_timestep > 0) or the CFL /
// corrector-controlled dt (d_timestep < 0), no SHTns, no inhomogeneous BC files.  The anelastic reference state (io.F90:559-608, the seven columns of
// planet_model.txt.in) is handed over by orc_set_reference_state.
//
// Build: g++ -O3 -march=native -fopenmp -ffp-contract=off -shared -fPIC
//        (oracle/build_oracle.sh).  -ffp-contract=off keeps a*b+c as two roundings, as
//        the reference's gfortran build without -ffp-contract does on x86 (no FMA).

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/lsd_b200.h"

namespace {

typedef std::complex<double> cplx;
const double d_PI = 3.1415926535897931;  // parameters.F90_template:263

// ----------------------------------------------------------------------------------------
// Band storage helpers.  mesh:   M(KL+1+n-j, j) = A(n,j), (2KL+1) x N  (meshs.F90:14-27)
//                        lumesh: M(2KL+1+n-j, j) = A(n,j), (3KL+1) x N, + ipiv
// ----------------------------------------------------------------------------------------
struct Band {
  int KL = 0, N = 0;
  std::vector<double> M;
  void init(int kl, int n) { KL = kl; N = n; M.assign((size_t)(2 * kl + 1) * n, 0.0); }
  double& at(int row, int col) { return M[(size_t)(row - 1) + (size_t)(2 * KL + 1) * (col - 1)]; }
  double at(int row, int col) const { return M[(size_t)(row - 1) + (size_t)(2 * KL + 1) * (col - 1)]; }
};
struct LUBand {
  int KL = 0, N = 0;
  std::vector<double> M;
  std::vector<int> ipiv;
  void init(int kl, int n) { KL = kl; N = n; M.assign((size_t)(3 * kl + 1) * n, 0.0); ipiv.assign(n, 0); }
  double& at(int row, int col) { return M[(size_t)(row - 1) + (size_t)(3 * KL + 1) * (col - 1)]; }
  double at(int row, int col) const { return M[(size_t)(row - 1) + (size_t)(3 * KL + 1) * (col - 1)]; }
};

// ---- LAPACK restatements --------------------------------------------------------------
// dgbtrf for KL=KU, unblocked path dgbtf2 (ILAENV's NB=32 > KL selects it).
int dgbtf2(int n, int kl, int ku, double* ab, int ldab, int* ipiv) {
  auto AB = [&](int i, int j) -> double& { return ab[(size_t)(i - 1) + (size_t)ldab * (j - 1)]; };
  int kv = ku + kl, info = 0;
  for (int j = ku + 2; j <= std::min(kv, n); ++j)
    for (int i = kv - j + 2; i <= kl; ++i) AB(i, j) = 0.0;
  int ju = 1;
  for (int j = 1; j <= n; ++j) {
    if (j + kv <= n)
      for (int i = 1; i <= kl; ++i) AB(i, j + kv) = 0.0;
    int km = std::min(kl, n - j);
    // idamax over AB(kv+1 .. kv+1+km, j): first index of maximal |.|
    int jp = 1;
    double amax = std::fabs(AB(kv + 1, j));
    for (int i = 2; i <= km + 1; ++i) {
      double v = std::fabs(AB(kv + i, j));
      if (v > amax) { amax = v; jp = i; }
    }
    ipiv[j - 1] = jp + j - 1;
    if (AB(kv + jp, j) != 0.0) {
      ju = std::max(ju, std::min(j + ku + jp - 1, n));
      if (jp != 1) {  // dswap(ju-j+1, AB(kv+jp,j), ldab-1, AB(kv+1,j), ldab-1)
        for (int c = 0; c <= ju - j; ++c) {
          double* a = &AB(kv + jp - c, j + c);
          double* b = &AB(kv + 1 - c, j + c);
          double t = *a; *a = *b; *b = t;
        }
      }
      if (km > 0) {
        double rp = 1.0 / AB(kv + 1, j);
        for (int i = 1; i <= km; ++i) AB(kv + 1 + i, j) *= rp;
        if (ju > j) {  // dger(km, ju-j, -1, AB(kv+2,j),1, AB(kv,j+1),ldab-1, AB(kv+1,j+1),ldab-1)
          for (int c = 1; c <= ju - j; ++c) {
            double y = AB(kv + 1 - c, j + c);
            if (y != 0.0) {
              double temp = -y;
              for (int i = 1; i <= km; ++i) AB(kv + 1 - c + i, j + c) += AB(kv + 1 + i, j) * temp;
            }
          }
        }
      }
    } else if (info == 0) {
      info = j;
    }
  }
  return info;
}

// dgbtrs('N', n, kl, ku, 1, ab, ldab, ipiv, b, n): forward with L and interchanges, then
// dtbsv upper non-unit (reference BLAS loop order).
void dgbtrs1(int n, int kl, int ku, const double* ab, int ldab, const int* ipiv, double* b) {
  auto AB = [&](int i, int j) -> double { return ab[(size_t)(i - 1) + (size_t)ldab * (j - 1)]; };
  int kd = ku + kl + 1;
  if (kl > 0) {
    for (int j = 1; j <= n - 1; ++j) {
      int lm = std::min(kl, n - j);
      int l = ipiv[j - 1];
      if (l != j) { double t = b[l - 1]; b[l - 1] = b[j - 1]; b[j - 1] = t; }
      double y = b[j - 1];
      if (y != 0.0) {
        double temp = -y;
        for (int i = 1; i <= lm; ++i) b[j + i - 1] += AB(kd + i, j) * temp;
      }
    }
  }
  int k = kl + ku, kplus1 = k + 1;
  for (int j = n; j >= 1; --j) {
    if (b[j - 1] != 0.0) {
      int l = kplus1 - j;
      b[j - 1] = b[j - 1] / AB(kplus1, j);
      double temp = b[j - 1];
      for (int i = j - 1; i >= std::max(1, j - k); --i) b[i - 1] -= temp * AB(l + i, j);
    }
  }
}

// dgetrf (unblocked dgetf2) + dgetri (unblocked, via dtrti2) for small n, lda.
int mat_invert(int n, double* a, int lda) {
  auto A = [&](int i, int j) -> double& { return a[(size_t)(i - 1) + (size_t)lda * (j - 1)]; };
  std::vector<int> ipiv(n);
  const double sfmin = 2.2250738585072014e-308;
  for (int j = 1; j <= n; ++j) {
    int jp = j;
    double amax = std::fabs(A(j, j));
    for (int i = j + 1; i <= n; ++i)
      if (std::fabs(A(i, j)) > amax) { amax = std::fabs(A(i, j)); jp = i; }
    ipiv[j - 1] = jp;
    if (A(jp, j) == 0.0) return j;
    if (jp != j)
      for (int c = 1; c <= n; ++c) { double t = A(j, c); A(j, c) = A(jp, c); A(jp, c) = t; }
    if (j < n) {
      if (std::fabs(A(j, j)) >= sfmin) {
        double r = 1.0 / A(j, j);
        for (int i = j + 1; i <= n; ++i) A(i, j) *= r;
      } else {
        for (int i = j + 1; i <= n; ++i) A(i, j) = A(i, j) / A(j, j);
      }
      for (int c = j + 1; c <= n; ++c) {
        double y = A(j, c);
        if (y != 0.0) {
          double temp = -y;
          for (int i = j + 1; i <= n; ++i) A(i, c) += A(i, j) * temp;
        }
      }
    }
  }
  // dtrti2: inverse of upper triangular U in place
  for (int j = 1; j <= n; ++j) {
    A(j, j) = 1.0 / A(j, j);
    double ajj = -A(j, j);
    // dtrmv('Upper','No transpose','Non-unit', j-1, A, lda, A(1,j), 1)
    for (int jj = 1; jj <= j - 1; ++jj) {
      double x = A(jj, j);
      if (x != 0.0) {
        double temp = x;
        for (int i = 1; i <= jj - 1; ++i) A(i, j) += temp * A(i, jj);
        A(jj, j) *= A(jj, jj);
      }
    }
    for (int i = 1; i <= j - 1; ++i) A(i, j) *= ajj;
  }
  // dgetri unblocked: solve inv(A)*L = inv(U)
  std::vector<double> work(n);
  for (int j = n; j >= 1; --j) {
    for (int i = j + 1; i <= n; ++i) { work[i - 1] = A(i, j); A(i, j) = 0.0; }
    if (j < n) {
      // dgemv('N', n, n-j, -1, A(1,j+1), lda, work(j+1), 1, 1, A(1,j), 1)
      for (int c = j + 1; c <= n; ++c) {
        double temp = -work[c - 1];
        if (work[c - 1] != 0.0)
          for (int i = 1; i <= n; ++i) A(i, j) += temp * A(i, c);
      }
    }
  }
  for (int j = n - 1; j >= 1; --j) {
    int jp = ipiv[j - 1];
    if (jp != j)
      for (int i = 1; i <= n; ++i) { double t = A(i, j); A(i, j) = A(i, jp); A(i, jp) = t; }
  }
  return 0;
}

// ---- FFT (restating FFTW's unnormalised DFT contract) ---------------------------------
struct FFTPlan {
  int n = 0;
  std::vector<int> factors;
  std::vector<cplx> wf, wb;  // e^{-2 pi i k/n}, e^{+2 pi i k/n}
  void init(int nn) {
    n = nn;
    factors.clear();
    int m = n;
    while (m % 4 == 0) { factors.push_back(4); m /= 4; }
    while (m % 2 == 0) { factors.push_back(2); m /= 2; }
    while (m % 3 == 0) { factors.push_back(3); m /= 3; }
    while (m % 5 == 0) { factors.push_back(5); m /= 5; }
    for (int p = 7; m > 1; p += 2)
      while (m % p == 0) { factors.push_back(p); m /= p; }
    wf.resize(n); wb.resize(n);
    for (int k = 0; k < n; ++k) {
      double a = 2.0 * d_PI * (double)k / (double)n;
      wf[k] = cplx(std::cos(a), -std::sin(a));
      wb[k] = std::conj(wf[k]);
    }
  }
  // recursive decimation in time: out[k] = sum_j in[j*stride] w^{jk}
  void rec(const cplx* in, cplx* out, int len, int stride, int fi, const std::vector<cplx>& w,
           cplx* scratch) const {
    if (len == 1) { out[0] = in[0]; return; }
    int p = factors[fi], m = len / p;
    for (int q = 0; q < p; ++q) rec(in + q * stride, out + q * m, m, stride * p, fi + 1, w, scratch);
    int tw = n / len;  // twiddle step
    for (int k = 0; k < m; ++k) {
      cplx t[16];
      for (int q = 0; q < p; ++q) t[q] = out[q * m + k] * w[(size_t)(q * k * tw) % n];
      for (int s = 0; s < p; ++s) {
        cplx acc = t[0];
        for (int q = 1; q < p; ++q) acc += t[q] * w[(size_t)(((q * s) % p) * (n / p))];
        scratch[s * m + k] = acc;
      }
    }
    for (int i = 0; i < len; ++i) out[i] = scratch[i];
  }
  void exec(const cplx* in, cplx* out, int sign, cplx* scratch) const {
    rec(in, out, n, 1, 0, sign < 0 ? wf : wb, scratch);
  }
};

// ---- fields -----------------------------------------------------------------------------
struct Coll {  // coll: Re(N, 0:H-1) column-major
  std::vector<double> re, im;
  void init(int N, int H) { re.assign((size_t)N * H, 0.0); im.assign((size_t)N * H, 0.0); }
};
struct Spec {  // spec: Re(0:H-1, N)
  std::vector<double> re, im;
  void init(int N, int H) { re.assign((size_t)N * H, 0.0); im.assign((size_t)N * H, 0.0); }
};
typedef std::vector<double> Phys;  // (Th, Ph, N)

struct RDom {
  int N = 0, KL = 0;
  std::vector<double> rp[7];  // r(n, p), p = -3..3
  std::vector<double> rho0, rho1, rho2, temp0, temp1, eta0, eta1;
  std::vector<double> intr2dr, f_factor;
  std::vector<double> intr2dr_comp, intr2dr_compS, intr2dr_magdiss, intr2dr_veldiss;
  std::vector<Band> dr;  // dr[1..KL]
  Band radLap, radLap_flayer, CompLap, GreLap, r1dr, compr1dr, MagTorLap, MagPolLap;
  double R(int n, int p) const { return rp[p + 3][n - 1]; }
};

}  // namespace

struct Oracle {
  lsd_config cfg;
  int L, M, Mp, N, KL, H, Th, Th2, Ph, Ma, Hc, Hr, Nic;
  std::vector<int> hl, hm, hs, thm;
  std::vector<double> ad_ll1, ad_ll11, ad_rtll1, ad_rtll11;
  std::vector<double> gp, gw, th, sn, sn1, gwP0;
  std::vector<double> P, P_, sin1mP, llP_, llsin1mP, qva, qvb, gwP, gwllP_, gwllsin1mP;
  RDom oc, ic;
  FFTPlan fft;
  // operators
  std::vector<LUBand> XTor, XPol, XGre, XC, XComp, mXTor, mXPol;
  std::vector<Band> YTor, YPol, YC, YComp, mYTor, mYPol;
  std::vector<double> Gre, invG;  // Gre(N,2,L) ; invG(2,2,L)
  // conducting inner core (Nic > 1): coupled field operators of size Nic + N - 1
  // (iclumesh), the inner core's Y bands, its field [Nic][H], nonlinear and saved terms
  std::vector<Band> icYTor, icYPol;
  Coll icTor, icPol, icNTor, icNPol, sv_icNTor, sv_icNPol;
  // inner-core rotation (rotation.F90; main.F90:92-94): rate, moment of inertia, the
  // torques of the last evaluation and the ones saved by rot_predictor / rot_corrector
  double rot_omega = 0, rot_inertia = 0, rot_velTorq = 0, rot_magTorq = 0, sv_velTorq = 0, sv_magTorq = 0;
  // state
  Coll vTor, vPol, codC, compC, bTor, bPol, bicTor, bicPol;
  // last nonlinear terms
  Coll vNTor, vNPol, codNC, compNC, bNTor, bNPol;
  // saved N (module-private NTor/NPol/NC of each field module)
  Coll sv_vNTor, sv_vNPol, sv_codNC, sv_compNC, sv_bNTor, sv_bNPol;
  // physical fields
  Phys vel_r, vel_t, vel_p, vel_cr, vel_ct, vel_cp, mag_r, mag_t, mag_p, mag_cr, mag_ct, mag_cp;
  Phys cod_gr, cod_gt, cod_gp, comp_gr, comp_gt, comp_gp;
  Phys vel_dur, vel_qv1, vel_dutr, vel_dupr, vel_qv2;  // anelastic (tra_qst2rtp_vel)
  // time
  double tim_t = 0, tim_dt = 0, tim_dterr = 0, tim_corr_dt = 0, tim_cfl_dt = 0, lasterr = 1e99;
  bool tim_new_dt = false;
  int tim_it = 0, tim_step = 0, tim_pcn = -1;
  int nthreads = 1;
  std::string err;
};

namespace {

// ========================================================================================
// Layout: parallel.h_template:54-100, variables.F90:103-194
// ========================================================================================
void setup_layout(Oracle& o) {
  o.hl.assign(o.H, 0); o.hm.assign(o.H, 0); o.hs.assign(o.H, 0);
  int nh = -1;
  for (int j = 1; j <= o.Hc; ++j) {        // _loop_setlm_begin with th_rnk = 0
    for (int i = 1; i <= o.Hr; ++i) {
      int m = j - 1;
      int l = m * o.Mp + i - 1;
      if (l >= o.L) { m = 2 * o.Hc - j; l = o.L - o.Hr + i - 1; }
      int m_ = m * o.Mp;
      ++nh;
      o.hl[nh] = l; o.hm[nh] = m_; o.hs[nh] = (l + m_) % 2;
    }
  }
  o.thm.assign(2 * o.Hc, 0);
  int m = -1, m_ = -1;                      // _loop_sumth_begin
  for (nh = 0; nh < o.H; ++nh) {
    int m__ = m_;
    m_ = o.hm[nh];
    if (m_ != m__) { ++m; o.thm[m] = m_ / o.Mp; }
  }
  o.ad_ll1.assign(o.L, 0); o.ad_ll11.assign(o.L, 0); o.ad_rtll1.assign(o.L, 0); o.ad_rtll11.assign(o.L, 0);
  for (int l = 1; l < o.L; ++l) {
    o.ad_ll1[l] = (double)(l * (l + 1));
    o.ad_ll11[l] = 1.0 / o.ad_ll1[l];
    o.ad_rtll1[l] = std::sqrt(o.ad_ll1[l]);
    o.ad_rtll11[l] = 1.0 / o.ad_rtll1[l];
  }
}

// ========================================================================================
// Gauss-Legendre points: auxiliary/gauwts.f:6-75
// ========================================================================================
void gauwts(double x1, double x2, double* gaux, double* gauw, int nthpts) {
  const double EPS = 1.0e-13, PI = 3.14159265358979312;
  int m = (nthpts + 1) / 2;
  double xm = 0.5 * (x2 + x1), xl = 0.5 * (x2 - x1);
  for (int i = 1; i <= m; ++i) {
    double z = std::cos(PI * ((double)i - 0.25) / ((double)nthpts + 0.5));
    double z1, pp;
    do {
      double p1 = 1.0, p2 = 0.0, p3;
      for (int j = 1; j <= nthpts; ++j) {
        p3 = p2; p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / (double)j;
      }
      pp = nthpts * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
    } while (std::fabs(z - z1) > EPS);
    gaux[i - 1] = xm - xl * z;
    gaux[nthpts - i] = xm + xl * z;
    gauw[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
    gauw[nthpts - i] = gauw[i - 1];
  }
}

// Schmidt-normalised P_l^m and dP/dtheta: auxiliary/schnla.f:21-115 with pmm.f, pmm1.f,
// plm.f, dpmm.f, dpmm1.f, dplm.f.  Index P_l^m -> pa[l(l+1)/2 + m].
double f_pmm(int m, double s) {
  if (m == 0) return 1.0;
  double p = std::sqrt(2.0);
  for (int i = 1; i <= m; ++i) { double twoi = 2.0 * i; p = p * s * std::sqrt((twoi - 1.0) / twoi); }
  return p;
}
double f_pmm1(int m, double x, double pmm0) { return x * pmm0 * std::sqrt(2.0 * m + 1.0); }
double f_plm(int l, int m, double x, double p1, double p2) {
  double rm = m, rl = l;
  double p = (2.0 * rl - 1.0) * x * p1;
  p = p - p2 * std::sqrt((rl + rm - 1.0) * (rl - rm - 1.0));
  return p / std::sqrt((rl + rm) * (rl - rm));
}
double f_dpmm(int m, double c, double s) {
  if (m == 0) return 0.0;
  double d = std::sqrt(2.0) * (double)m * c / s;
  for (int i = 1; i <= m; ++i) { double twoi = 2.0 * i; d = d * s * std::sqrt((twoi - 1.0) / twoi); }
  return d;
}
double f_dpmm1(int m, double x, double s, double pmm0, double dpmm0) {
  return std::sqrt(2.0 * m + 1.0) * (x * dpmm0 - s * pmm0);
}
double f_dplm(int l, int m, double x, double s, double p1, double d1, double d2) {
  double rm = m, rl = l;
  double d = (2.0 * rl - 1.0) * (x * d1 - s * p1);
  d = d - d2 * std::sqrt((rl + rm - 1.0) * (rl - rm - 1.0));
  return d / std::sqrt((rl + rm) * (rl - rm));
}
int schnla(double* pa, double* dpa, double x, int lh) {
  if (x * x > 1.0) return 1;
  double sine = std::sqrt((1.0 + x) * (1.0 - x));
  if (sine < 1.0e-6) return 2;
  auto IDX = [](int l, int m) { return l * (l + 1) / 2 + m; };
  for (int m = 0; m <= lh - 2; ++m) {
    int l = m;
    int index = IDX(l, m);
    pa[index] = f_pmm(m, sine);
    dpa[index] = f_dpmm(m, x, sine);
    double pmin1 = pa[index], dpmin1 = dpa[index];
    int iold2 = index;
    l = l + 1;
    index = IDX(l, m);
    pa[index] = f_pmm1(m, x, pmin1);
    dpa[index] = f_dpmm1(m, x, sine, pmin1, dpmin1);
    int iold1 = index;
    for (l = m + 2; l <= lh; ++l) {
      double pmin2 = pa[iold2]; pmin1 = pa[iold1];
      double dpmin2 = dpa[iold2]; dpmin1 = dpa[iold1];
      index = IDX(l, m);
      pa[index] = f_plm(l, m, x, pmin1, pmin2);
      dpa[index] = f_dplm(l, m, x, sine, pmin1, dpmin1, dpmin2);
      iold2 = iold1; iold1 = index;
    }
  }
  int m = lh - 1, l = m;
  int index = IDX(l, m);
  pa[index] = f_pmm(m, sine);
  dpa[index] = f_dpmm(m, x, sine);
  double pmin1 = pa[index], dpmin1 = dpa[index];
  l = lh;
  index = IDX(l, m);
  pa[index] = f_pmm1(m, x, pmin1);
  dpa[index] = f_dpmm1(m, x, sine, pmin1, dpmin1);
  m = lh;
  index = IDX(l, m);
  pa[index] = f_pmm(m, sine);
  dpa[index] = f_dpmm(m, x, sine);
  return 0;
}

// legendre.F90:63-128
int setup_legendre(Oracle& o) {
  o.gp.assign(o.Th, 0); o.gw.assign(o.Th, 0);
  gauwts(-1.0, 1.0, o.gp.data(), o.gw.data(), o.Th);
  o.th.resize(o.Th); o.sn.resize(o.Th); o.sn1.resize(o.Th); o.gwP0.assign(o.Th, 0);
  for (int j = 0; j < o.Th; ++j) {
    o.th[j] = std::acos(o.gp[j]);
    o.sn[j] = std::sin(o.th[j]);
    o.sn1[j] = 1.0 / o.sn[j];
  }
  size_t sz = (size_t)o.Th2 * o.H;
  for (auto* t : {&o.P, &o.P_, &o.sin1mP, &o.llP_, &o.llsin1mP, &o.qva, &o.qvb, &o.gwP, &o.gwllP_, &o.gwllsin1mP})
    t->assign(sz, 0.0);
  int L1 = o.L - 1;
  std::vector<double> pa((L1 + 1) * (L1 + 2) / 2), dpa((L1 + 1) * (L1 + 2) / 2);
  for (int j = 1; j <= o.Th2; ++j) {
    if (schnla(pa.data(), dpa.data(), o.gp[j - 1], L1) != 0) return 1;
    for (int nh = 0; nh < o.H; ++nh) {
      int l = o.hl[nh], m_ = o.hm[nh];
      int k = l * (l + 1) / 2 + m_;
      size_t id = (size_t)(j - 1) + (size_t)o.Th2 * nh;
      o.P[id] = pa[k];
      o.P_[id] = dpa[k];
      o.sin1mP[id] = pa[k] * m_ * o.sn1[j - 1];
      if (l == 0) {
        o.llP_[id] = 0.0; o.llsin1mP[id] = 0.0;
      } else {
        double w = 1.0 / std::sqrt((double)(l * (l + 1)));
        o.llP_[id] = dpa[k] * w;
        o.llsin1mP[id] = pa[k] * w * m_ * o.sn1[j - 1];
        o.qva[id] = o.llsin1mP[id] * (double)m_ * o.sn1[j - 1] - o.llP_[id] * o.gp[j - 1] * o.sn1[j - 1];
        o.qvb[id] = o.llsin1mP[id] * o.gp[j - 1] * o.sn1[j - 1] - o.llP_[id] * (double)m_ * o.sn1[j - 1];
      }
    }
    o.gwP0[j - 1] = pa[0] * o.gw[j - 1] * 0.5;
    o.gwP0[o.Th - j] = o.gwP0[j - 1];
  }
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh], m_ = o.hm[nh];
    int m = m_ / o.Mp;
    for (int j = 1; j <= o.Th2; ++j) {
      size_t id = (size_t)(j - 1) + (size_t)o.Th2 * nh;
      double w = o.gw[j - 1] * ((2.0 * l + 1.0) / 4.0);
      if (m == 0) w = 2.0 * w;
      o.gwP[id] = o.P[id] * w;
      if (l == 0) {
        o.gwllP_[id] = 0.0; o.gwllsin1mP[id] = 0.0;
      } else {
        w = w / std::sqrt((double)(l * (l + 1)));
        o.gwllP_[id] = o.P_[id] * w;
        o.gwllsin1mP[id] = o.P[id] * w * m_ * o.sn1[j - 1];
      }
    }
  }
  return 0;
}

// ========================================================================================
// Radial mesh: meshs.F90:116-419 (Boussinesq: rho = Temp0 = 0, eta = 1, deta = 0,
// io.F90:545-556 and the zero-initialised module storage)
// ========================================================================================
int rdom_init(RDom& D, int KL) {
  D.KL = KL;
  int N = D.N;
  for (int p = -3; p <= 3; ++p) {
    if (p == 1) continue;
    D.rp[p + 3].resize(N);
    for (int n = 0; n < N; ++n) {  // integer powers as products, like gfortran's r**p
      double x = D.rp[4][n], y = 1.0;
      for (int k = 0; k < (p < 0 ? -p : p); ++k) y = (k == 0) ? x : y * x;
      D.rp[p + 3][n] = p < 0 ? 1.0 / y : y;
    }
  }
  D.dr.resize(KL + 1);
  for (int i = 1; i <= KL; ++i) D.dr[i].init(KL, N);
  for (Band* b : {&D.radLap, &D.radLap_flayer, &D.CompLap, &D.GreLap, &D.r1dr, &D.compr1dr, &D.MagTorLap, &D.MagPolLap})
    b->init(KL, N);
  D.intr2dr.assign(N, 0.0);
  D.f_factor.assign(N, 0.0);
  for (auto* v : {&D.intr2dr_comp, &D.intr2dr_compS, &D.intr2dr_magdiss, &D.intr2dr_veldiss}) v->assign(N, 0.0);
  if (N == 1) return 0;
  const int lda = 2 * KL + 1;
  std::vector<double> A((size_t)lda * lda);
  auto Aa = [&](int i, int j) -> double& { return A[(size_t)(i - 1) + (size_t)lda * (j - 1)]; };
  for (int n = 1; n <= N; ++n) {
    int l = std::max(1, n - KL), r = std::min(n + KL, N), nn = r - l + 1;
    for (int i = 1; i <= nn; ++i) Aa(i, 1) = 1.0;
    for (int j = 2; j <= nn; ++j)
      for (int i = 1; i <= nn; ++i)
        Aa(i, j) = Aa(i, j - 1) * (D.R(l + i - 1, 1) - D.R(n, 1)) / (double)(j - 1);
    if (mat_invert(nn, A.data(), lda) != 0) return 1;
    for (int i = 1; i <= KL; ++i)
      for (int j = l; j <= r; ++j) D.dr[i].at(KL + 1 + n - j, j) = Aa(i + 1, j - l + 1);
    double c = 1.0, e = 1.0;
    for (int i = 1; i <= nn; ++i) {
      c = c * (D.R(std::min(n + 1, N), 1) - D.R(n, 1)) / (double)i;
      e = e * (D.R(std::max(1, n - 1), 1) - D.R(n, 1)) / (double)i;
      for (int j = l; j <= r; ++j) {
        double w = 0.5 * (c - e) * Aa(i, j - l + 1) * D.R(n, 2);
        D.intr2dr[j - 1] = D.intr2dr[j - 1] + w;
        // the density / temperature / diffusivity weighted weights (meshs.F90:318-333)
        D.intr2dr_comp[j - 1] = D.intr2dr_comp[j - 1] + w * D.rho0[n - 1];
        D.intr2dr_compS[j - 1] = D.intr2dr_compS[j - 1] + w * (D.rho0[n - 1] * D.temp0[n - 1]);
        D.intr2dr_magdiss[j - 1] = D.intr2dr_magdiss[j - 1] + w * D.eta0[n - 1];
        D.intr2dr_veldiss[j - 1] = D.intr2dr_veldiss[j - 1] +
                                   w * 2.0 * D.rho0[n - 1] * (D.rho2[n - 1] - D.rho1[n - 1] * D.rho1[n - 1] / 3.0);
      }
    }
  }
  for (int j = 1; j <= N; ++j) {
    int l = std::max(1, j - KL), r = std::min(j + KL, N);
    for (int n = l; n <= r; ++n)
      D.radLap.at(KL + 1 + n - j, j) = D.dr[2].at(KL + 1 + n - j, j) + D.dr[1].at(KL + 1 + n - j, j) * 2.0 * D.R(n, -1);
  }
  const double d_flayer_radius = -1.0, d_transition_width = (double)0.05f, d_enhance_diff = 1.0;
  for (int j = 1; j <= N; ++j) {
    double ss = 0.5 + 0.5 * std::tanh((D.R(j, 1) - d_flayer_radius) / d_transition_width);
    double cc = ss + (1 - ss) * d_enhance_diff;
    D.f_factor[j - 1] = cc;
    int l = std::max(1, j - KL), r = std::min(j + KL, N);
    for (int n = l; n <= r; ++n)
      D.radLap_flayer.at(KL + 1 + n - j, j) =
          cc * (D.dr[2].at(KL + 1 + n - j, j) + D.dr[1].at(KL + 1 + n - j, j) * 2.0 * D.R(n, -1));
  }
  for (int j = 1; j <= N; ++j) {
    int l = std::max(1, j - KL), r = std::min(j + KL, N);
    for (int n = l; n <= r; ++n) {
      int row = KL + 1 + n - j;
      D.CompLap.at(row, j) = D.dr[2].at(row, j) + 2.0 * (D.rho1[n - 1] + D.R(n, -1)) * D.dr[1].at(row, j);
      D.MagTorLap.at(row, j) = D.eta0[n - 1] * (D.dr[2].at(row, j) + 2.0 * D.R(n, -1) * D.dr[1].at(row, j)) +
                               D.eta1[n - 1] * D.dr[1].at(row, j);
      D.MagPolLap.at(row, j) = D.eta0[n - 1] * (D.dr[2].at(row, j) + 2.0 * D.R(n, -1) * D.dr[1].at(row, j));
    }
  }
  for (int j = 1; j <= N; ++j) {
    int l = std::max(1, j - KL), r = std::min(j + KL, N);
    for (int n = l; n <= r; ++n) {
      int row = KL + 1 + n - j;
      D.GreLap.at(row, j) = D.dr[2].at(row, j) + (D.rho1[n - 1] + 2.0 * D.R(n, -1)) * D.dr[1].at(row, j);
    }
  }
  D.r1dr.M = D.dr[1].M;
  D.compr1dr.M = D.dr[1].M;
  for (int j = 1; j <= N; ++j) {
    D.r1dr.at(KL + 1, j) = D.r1dr.at(KL + 1, j) + D.R(j, -1);
    D.compr1dr.at(KL + 1, j) = D.compr1dr.at(KL + 1, j) + D.R(j, -1) + D.rho1[j - 1];
  }
  return 0;
}

int setup_mesh(Oracle& o) {
  RDom& D = o.oc;
  D.N = o.N;
  D.rp[4].resize(o.N);
  for (int n = 1; n <= o.N; ++n) {
    if (o.cfg.alpha > 0)
      D.rp[4][n - 1] = 0.5 * (1.0 + std::asin(o.cfg.alpha * std::cos(d_PI * (o.N - n) / (double)(o.N - 1))) / std::asin(o.cfg.alpha));
    else
      D.rp[4][n - 1] = 0.5 * (1.0 + std::cos(d_PI * (o.N - n) / (double)(o.N - 1)));
  }
  double ri = o.cfg.rratio / (1.0 - o.cfg.rratio);
  for (int n = 0; n < o.N; ++n) D.rp[4][n] = D.rp[4][n] + ri;
  for (auto* v : {&D.rho0, &D.rho1, &D.rho2, &D.temp0, &D.temp1}) v->assign(o.N, 0.0);
  D.eta0.assign(o.N, 1.0); D.eta1.assign(o.N, 0.0);
  if (!o.cfg.boussinesq) {  // until orc_set_reference_state: rho = T = 1, gradients 0
    D.rho0.assign(o.N, 1.0); D.temp0.assign(o.N, 1.0);
  }
  RDom& I = o.ic;
  I.N = o.Nic;
  I.rp[4].resize(o.Nic);
  int N_ = 2 * o.Nic;
  for (int n = o.Nic + 1; n <= N_; ++n) I.rp[4][n - o.Nic - 1] = ri * std::cos(d_PI * (N_ - n) / (double)(N_ - 1));
  for (auto* v : {&I.rho0, &I.rho1, &I.rho2, &I.temp0, &I.temp1}) v->assign(o.Nic, 0.0);
  I.eta0.assign(o.Nic, 1.0); I.eta1.assign(o.Nic, 0.0);
  if (rdom_init(D, o.KL)) return 1;
  if (rdom_init(I, o.KL)) return 1;
  return 0;
}

// ========================================================================================
// Operators: timestep.F90:47-546, velocity.F90:56-273, codensity.F90:37-119,
// composition.F90 (clone), magnetic.F90:62-282
// ========================================================================================
void lumesh_from_band(LUBand& A, const Band& B, double fac) {  // A%M(KL+1:,:) = fac*B%M
  int KL = A.KL;
  for (int j = 1; j <= A.N; ++j)
    for (int row = 1; row <= 2 * KL + 1; ++row) A.at(KL + row, j) = fac * B.at(row, j);
}
void lumesh_zero_bc_rows(LUBand& A) {
  int KL = A.KL, N = A.N;
  for (int j = 1; j <= 1 + KL; ++j) A.at(2 * KL + 1 + 1 - j, j) = 0.0;
  for (int j = N - KL; j <= N; ++j) A.at(2 * KL + 1 + N - j, j) = 0.0;
}
// tim_lumesh_flayer_X (timestep.F90:175-208) -- the Boussinesq velocity operator
void tim_lumesh_flayer_X(const Oracle& o, const RDom& D, double c1, double c2, int l, LUBand& A) {
  double c1_ = c1 / o.tim_dt, c2_ = c2 * o.cfg.implicit;
  if (o.cfg.implicit == 0.0) c2_ = 1.0;
  double ll1 = (double)(l * (l + 1));
  A.init(o.KL, D.N);
  lumesh_from_band(A, D.radLap_flayer, -c2_);
  for (int n = 1; n <= D.N; ++n) {
    double t = ll1 * D.R(n, -2);
    A.at(2 * o.KL + 1, n) = A.at(2 * o.KL + 1, n) + c1_ + c2_ * (t + o.cfg.Hyp * t * t) * D.f_factor[n - 1];
  }
  lumesh_zero_bc_rows(A);
}
// tim_lumesh_X (timestep.F90:138-169) -- codensity / composition operator
void tim_lumesh_X(const Oracle& o, const RDom& D, double c1, double c2, int l, LUBand& A) {
  double c1_ = c1 / o.tim_dt, c2_ = c2 * o.cfg.implicit;
  if (o.cfg.implicit == 0.0) c2_ = 1.0;
  double ll1 = (double)(l * (l + 1));
  A.init(o.KL, D.N);
  lumesh_from_band(A, D.GreLap, -c2_);
  for (int n = 1; n <= D.N; ++n) {
    double t = ll1 * D.R(n, -2);
    A.at(2 * o.KL + 1, n) = A.at(2 * o.KL + 1, n) + c1_ + c2_ * (t + o.cfg.Hyp * t * t);
  }
  lumesh_zero_bc_rows(A);
}
// tim_iclumesh_Tor_X / _Pol_X with Ni = 1, Boussinesq (timestep.F90:214-344)
void tim_iclumesh_X(const Oracle& o, const RDom& D, double c1, double c2, int l, bool tor, LUBand& A) {
  double c1_ = c1 / o.tim_dt, c2_ = c2 * o.cfg.implicit;
  if (o.cfg.implicit == 0.0) c2_ = 1.0;
  double ll1 = (double)(l * (l + 1));
  A.init(o.KL, D.N);
  const Band& lap = tor ? D.MagTorLap : D.MagPolLap;
  for (int j = 1; j <= A.N; ++j)
    for (int row = 1; row <= 2 * o.KL + 1; ++row) A.at(o.KL + row, j) = A.at(o.KL + row, j) - c2_ * lap.at(row, j);
  for (int n = 1; n <= D.N; ++n)
    A.at(2 * o.KL + 1, n) = A.at(2 * o.KL + 1, n) + c1_ + c2_ * ll1 * D.R(n, -2);
  lumesh_zero_bc_rows(A);
}
// tim_iclumesh_Tor_X / _Pol_X with a conducting inner core (Ni > 1), Boussinesq
// (timestep.F90:218-344), and the rows of mag_bc_Tor / mag_bc_Pol (magnetic.F90:137-282):
// unknowns 1..Ni on the inner-core mesh, Ni..Ni+No-1 on the outer-core mesh (point Ni,
// the inner-core boundary, shared); row 1 regularity at the innermost point, row Ni the
// continuity of dr across the boundary, row Ni+No-1 the insulating exterior.
void tim_iclumesh_X_cic(const Oracle& o, double c1, double c2, int l, bool tor, LUBand& A) {
  const RDom& I = o.ic;
  const RDom& D = o.oc;
  const int KL = o.KL, Ni = I.N, No = D.N, N_ = Ni + No - 1;
  double c1_ = c1 / o.tim_dt, c2_ = c2 * o.cfg.implicit;
  if (o.cfg.implicit == 0.0) c2_ = 1.0;
  const double ll1 = (double)(l * (l + 1));
  A.init(KL, N_);
  for (int j = 1; j <= Ni; ++j)
    for (int row = 1; row <= 2 * KL + 1; ++row) A.at(KL + row, j) = -c2_ * I.radLap.at(row, j);
  for (int n = 1; n <= Ni; ++n) A.at(2 * KL + 1, n) = A.at(2 * KL + 1, n) + c1_ + c2_ * ll1 * I.R(n, -2);
  const Band& lap = tor ? D.MagTorLap : D.MagPolLap;
  for (int j = 1; j <= No; ++j)
    for (int row = 1; row <= 2 * KL + 1; ++row)
      A.at(KL + row, j + Ni - 1) = A.at(KL + row, j + Ni - 1) - c2_ * lap.at(row, j);
  for (int n = 1; n <= No; ++n)
    A.at(2 * KL + 1, n + Ni - 1) = A.at(2 * KL + 1, n + Ni - 1) + c1_ + c2_ * ll1 * D.R(n, -2);
  for (int j = 1; j <= 1 + KL; ++j) A.at(2 * KL + 1 + 1 - j, j) = 0.0;
  for (int j = N_ - KL; j <= N_; ++j) A.at(2 * KL + 1 + N_ - j, j) = 0.0;
  for (int j = Ni - KL; j <= Ni + KL; ++j) A.at(2 * KL + 1 + Ni - j, j) = 0.0;
  if (tor) {  // BTor = 0 at the innermost point and outside
    A.at(2 * KL + 1, 1) = 1.0;
    A.at(2 * KL + 1, N_) = 1.0;
  } else {  // (dr - l/r) BPol = 0 innermost, (dr + (l+1)/r) BPol = 0 at the outer wall
    for (int j = 1; j <= 1 + KL; ++j) A.at(2 * KL + 1 + 1 - j, j) = I.dr[1].at(KL + 1 + 1 - j, j);
    A.at(2 * KL + 1, 1) = A.at(2 * KL + 1, 1) - I.R(1, -1) * l;
    for (int j = No - KL; j <= No; ++j) {
      const int j_ = j + Ni - 1;
      A.at(2 * KL + 1 + N_ - j_, j_) = D.dr[1].at(KL + 1 + No - j, j);
    }
    A.at(2 * KL + 1, N_) = A.at(2 * KL + 1, N_) + D.R(No, -1) * (l + 1);
  }
  for (int j = 2; j <= 1 + KL; ++j) {  // dr continuous across the inner-core boundary
    const int j_ = j + Ni - 1;
    A.at(2 * KL + 1 + Ni - j_, j_) = D.dr[1].at(KL + 1 + 1 - j, j);
  }
  for (int j = Ni - KL; j <= Ni - 1; ++j) A.at(2 * KL + 1 + Ni - j, j) = -I.dr[1].at(KL + 1 + Ni - j, j);
  A.at(2 * KL + 1, Ni) = D.dr[1].at(KL + 1, 1) - I.dr[1].at(KL + 1, Ni);
}
// tim_lumesh_vel_X (timestep.F90:47-86) -- the anelastic velocity operator
void tim_lumesh_vel_X(const Oracle& o, const RDom& D, double c1, double c2, int l, LUBand& A) {
  double c1_ = c1 / o.tim_dt, c2_ = c2 * o.cfg.implicit;
  if (o.cfg.implicit == 0.0) c2_ = 1.0;
  double ll1 = (double)(l * (l + 1));
  A.init(o.KL, D.N);
  lumesh_from_band(A, D.CompLap, -c2_);
  for (int n = 1; n <= D.N; ++n) {
    double t = ll1 * D.R(n, -2), x1 = D.rho1[n - 1];
    double d = t + o.cfg.Hyp * (t * t);
    d = d - 2.0 * x1 * D.R(n, -1);
    d = d - x1 * x1;
    d = d - D.rho2[n - 1];
    A.at(2 * o.KL + 1, n) = A.at(2 * o.KL + 1, n) + c1_ + c2_ * d;
  }
  lumesh_zero_bc_rows(A);
}
// tim_lumesh_Gre_X (timestep.F90:92-128) -- the anelastic Green's function operator
void tim_lumesh_Gre_X(const Oracle& o, const RDom& D, double c1, double c2, int l, LUBand& A) {
  double c1_ = c1 / o.tim_dt, c2_ = c2 * o.cfg.implicit;
  if (o.cfg.implicit == 0.0) c2_ = 1.0;
  double ll1 = (double)(l * (l + 1));
  A.init(o.KL, D.N);
  lumesh_from_band(A, D.GreLap, -c2_);
  for (int n = 1; n <= D.N; ++n) {
    double d = ll1 * D.R(n, -2) - D.rho1[n - 1] * D.R(n, -1);
    d = d - D.rho2[n - 1];
    A.at(2 * o.KL + 1, n) = A.at(2 * o.KL + 1, n) + c1_ + c2_ * d;
  }
  lumesh_zero_bc_rows(A);
}
// tim_iclumesh_Tor_X / _Pol_X with Ni = 1, anelastic diagonal (timestep.F90:243-262, 311-322)
void tim_iclumesh_X_anel(const Oracle& o, const RDom& D, double c1, double c2, int l, bool tor, LUBand& A) {
  double c1_ = c1 / o.tim_dt, c2_ = c2 * o.cfg.implicit;
  if (o.cfg.implicit == 0.0) c2_ = 1.0;
  double ll1 = (double)(l * (l + 1));
  A.init(o.KL, D.N);
  const Band& lap = tor ? D.MagTorLap : D.MagPolLap;
  for (int j = 1; j <= A.N; ++j)
    for (int row = 1; row <= 2 * o.KL + 1; ++row) A.at(o.KL + row, j) = A.at(o.KL + row, j) - c2_ * lap.at(row, j);
  for (int n = 1; n <= D.N; ++n) {
    double t = ll1 * D.R(n, -2);
    double d = ll1 * D.eta0[n - 1] * D.R(n, -2);
    if (tor) d = d - D.eta1[n - 1] * D.R(n, -1);
    d = d + o.cfg.Hyp * (t * t);
    A.at(2 * o.KL + 1, n) = A.at(2 * o.KL + 1, n) + c1_ + c2_ * d;
  }
  lumesh_zero_bc_rows(A);
}
// tim_mesh_vel_Y (timestep.F90:350-380)
void tim_mesh_vel_Y(const Oracle& o, const RDom& D, double c1, double c2, int l, Band& A) {
  double c1_ = c1 / o.tim_dt, c2_ = c2 * (1.0 - o.cfg.implicit);
  A.init(o.KL, D.N);
  for (size_t i = 0; i < A.M.size(); ++i) A.M[i] = c2_ * D.CompLap.M[i];
  for (int n = 1; n <= D.N; ++n) {
    double t = (double)(l * (l + 1)) * D.R(n, -2), x1 = D.rho1[n - 1];
    double d = t + o.cfg.Hyp * (t * t);
    d = d - 2.0 * x1 * D.R(n, -1);
    d = d - x1 * x1;
    d = d - D.rho2[n - 1];
    A.at(o.KL + 1, n) = A.at(o.KL + 1, n) + c1_ - c2_ * d;
  }
}
// tim_mesh_mag_Tor_Y / _Pol_Y (timestep.F90:466-546)
void tim_mesh_mag_Y(const Oracle& o, const RDom& D, double c1, double c2, int l, bool tor, Band& A) {
  double c1_ = c1 / o.tim_dt, c2_ = c2 * (1.0 - o.cfg.implicit);
  A.init(o.KL, D.N);
  const Band& lap = tor ? D.MagTorLap : D.MagPolLap;
  for (size_t i = 0; i < A.M.size(); ++i) A.M[i] = c2_ * lap.M[i];
  for (int n = 1; n <= D.N; ++n) {
    double t = (double)(l * (l + 1)) * D.R(n, -2);
    double d = (double)(l * (l + 1)) * D.eta0[n - 1] * D.R(n, -2);
    if (tor) d = d - D.eta1[n - 1] * D.R(n, -1);
    d = d + o.cfg.Hyp * (t * t);
    A.at(o.KL + 1, n) = A.at(o.KL + 1, n) + c1_ - c2_ * d;
  }
}
// tim_mesh_flayer_Y (timestep.F90:442-458)
void tim_mesh_flayer_Y(const Oracle& o, const RDom& D, double c1, double c2, int l, Band& A) {
  double c1_ = c1 / o.tim_dt, c2_ = c2 * (1.0 - o.cfg.implicit);
  A.init(o.KL, D.N);
  for (size_t i = 0; i < A.M.size(); ++i) A.M[i] = c2_ * D.radLap_flayer.M[i];
  for (int n = 1; n <= D.N; ++n) {
    double t = (double)(l * (l + 1)) * D.R(n, -2);
    A.at(o.KL + 1, n) = A.at(o.KL + 1, n) + c1_ - c2_ * (t + o.cfg.Hyp * t * t) * D.f_factor[n - 1];
  }
}
// tim_mesh_Y (timestep.F90:416-436)
void tim_mesh_Y(const Oracle& o, const RDom& D, double c1, double c2, int l, Band& A) {
  double c1_ = c1 / o.tim_dt, c2_ = c2 * (1.0 - o.cfg.implicit);
  A.init(o.KL, D.N);
  for (size_t i = 0; i < A.M.size(); ++i) A.M[i] = c2_ * D.GreLap.M[i];
  for (int n = 1; n <= D.N; ++n) {
    double t = (double)(l * (l + 1)) * D.R(n, -2);
    A.at(o.KL + 1, n) = A.at(o.KL + 1, n) + c1_ - c2_ * (t + o.cfg.Hyp * t * t);
  }
}

int lu_find(LUBand& A) {
  return dgbtf2(A.N, A.KL, A.KL, A.M.data(), 3 * A.KL + 1, A.ipiv.data());
}

// tim_invX (timestep.F90:566-588) on a coll
void tim_invX(const Oracle& o, bool zero, const std::vector<LUBand>& A, Coll& b) {
  int N = o.N;
#pragma omp parallel for schedule(static)
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh];
    if (l == 0 && !zero) continue;
    dgbtrs1(N, o.KL, o.KL, A[l].M.data(), 3 * o.KL + 1, A[l].ipiv.data(), &b.re[(size_t)N * nh]);
    dgbtrs1(N, o.KL, o.KL, A[l].M.data(), 3 * o.KL + 1, A[l].ipiv.data(), &b.im[(size_t)N * nh]);
  }
}
// tim_icinvX (timestep.F90:594-634): the coupled solve, b = (ic rows 1..Ni-1, oc rows)
void tim_icinvX(const Oracle& o, const std::vector<LUBand>& A, Coll& oc, Coll& ic) {
  const int Ni = o.Nic, No = o.N, N_ = Ni + No - 1;
#pragma omp parallel for schedule(static)
  for (int nh = 0; nh < o.H; ++nh) {
    if (o.hl[nh] == 0) continue;
    std::vector<double> b(N_);
    for (int part = 0; part < 2; ++part) {
      double* icv = part == 0 ? &ic.re[(size_t)Ni * nh] : &ic.im[(size_t)Ni * nh];
      double* ocv = part == 0 ? &oc.re[(size_t)No * nh] : &oc.im[(size_t)No * nh];
      for (int n = 0; n < Ni - 1; ++n) b[n] = icv[n];
      for (int n = 0; n < No; ++n) b[Ni - 1 + n] = ocv[n];
      dgbtrs1(N_, o.KL, o.KL, A[o.hl[nh]].M.data(), 3 * o.KL + 1, A[o.hl[nh]].ipiv.data(), b.data());
      for (int n = 0; n < Ni; ++n) icv[n] = b[n];
      for (int n = 0; n < No; ++n) ocv[n] = b[Ni - 1 + n];
    }
  }
}
// tim_multY (timestep.F90:640-670): d = A b + c, columns of N rows
void tim_multY_n(const Oracle& o, int N, bool zero, const std::vector<Band>& A, const Coll& b, const Coll& c,
                 Coll& d);
void tim_multY(const Oracle& o, bool zero, const std::vector<Band>& A, const Coll& b, const Coll& c, Coll& d) {
  tim_multY_n(o, o.N, zero, A, b, c, d);
}
void tim_multY_n(const Oracle& o, int N, bool zero, const std::vector<Band>& A, const Coll& b, const Coll& c,
                 Coll& d) {
  int KL = o.KL;
  if (&d != &c) d = c;
#pragma omp parallel for schedule(static)
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh];
    if (l == 0 && !zero) continue;
    double* dr = &d.re[(size_t)N * nh];
    double* di = &d.im[(size_t)N * nh];
    const double* br = &b.re[(size_t)N * nh];
    const double* bi = &b.im[(size_t)N * nh];
    for (int j = 1; j <= N; ++j) {
      int nl = std::max(1, j - KL), nr = std::min(j + KL, N);
      for (int n = nl; n <= nr; ++n) {
        dr[n - 1] = dr[n - 1] + A[l].at(KL + 1 + n - j, j) * br[j - 1];
        di[n - 1] = di[n - 1] + A[l].at(KL + 1 + n - j, j) * bi[j - 1];
      }
    }
  }
}
void tim_zerobc_n(const Oracle& o, int N, Coll& a) {
  for (int nh = 0; nh < o.H; ++nh) {
    a.re[(size_t)N * nh] = 0.0; a.re[(size_t)N * nh + N - 1] = 0.0;
    a.im[(size_t)N * nh] = 0.0; a.im[(size_t)N * nh + N - 1] = 0.0;
  }
}
void tim_zerobc(const Oracle& o, Coll& a) { tim_zerobc_n(o, o.N, a); }
void tim_nlincorr(const Oracle& o, const Coll& n, const Coll& np, Coll& nc) {
  double c = o.cfg.implicit;
  nc.re.resize(n.re.size()); nc.im.resize(n.im.size());
  for (size_t i = 0; i < n.re.size(); ++i) {
    nc.re[i] = c * (n.re[i] - np.re[i]);
    nc.im[i] = c * (n.im[i] - np.im[i]);
  }
}
void tim_addcorr(Oracle& o, const Coll& ac, Coll& a, int nrows, int N) {
  // nrows = a%D%N (columns of stride N); for the ic fields with Ni = 1 only row 1
  double dterr = 0.0;
  for (int nh = 0; nh < o.H; ++nh)
    for (int n = 0; n < nrows; ++n) {
      size_t i = (size_t)N * nh + n;
      dterr = dterr + ac.re[i] * ac.re[i];
      dterr = dterr + ac.im[i] * ac.im[i];
      a.re[i] = a.re[i] + ac.re[i];
      a.im[i] = a.im[i] + ac.im[i];
    }
  o.tim_dterr = o.tim_dterr + std::sqrt(dterr);
}

int build_matrices(Oracle& o) {
  const RDom& D = o.oc;
  int L = o.L, KL = o.KL, N = o.N;
  o.XTor.assign(L, LUBand()); o.XPol.assign(L, LUBand()); o.XGre.assign(L, LUBand());
  o.YTor.assign(L, Band()); o.YPol.assign(L, Band());
  o.XC.assign(L, LUBand()); o.YC.assign(L, Band()); o.XComp.assign(L, LUBand()); o.YComp.assign(L, Band());
  o.mXTor.assign(L, LUBand()); o.mXPol.assign(L, LUBand()); o.mYTor.assign(L, Band()); o.mYPol.assign(L, Band());
  int bad = 0;
  // vel_matrices (velocity.F90:56-168); Boussinesq uses the flayer operators, the
  // anelastic equations tim_lumesh_vel_X / tim_mesh_vel_Y / tim_lumesh_Gre_X
  const bool bq = o.cfg.boussinesq != 0;
  double c1 = 1.0, c2 = o.cfg.Pm;
  for (int l = 1; l < L; ++l) {
    if (bq) tim_lumesh_flayer_X(o, D, c1, c2, l, o.XTor[l]);
    else tim_lumesh_vel_X(o, D, c1, c2, l, o.XTor[l]);
    // vel_bc_Tor (velocity.F90:177-201)
    LUBand& A = o.XTor[l];
    if (o.cfg.vel_bc == 1 || o.cfg.vel_bc == 2) {
      A.at(2 * KL + 1, 1) = 1.0;
    } else {
      for (int j = 1; j <= 1 + KL; ++j) A.at(2 * KL + 1 + 1 - j, j) = D.dr[1].at(KL + 1 + 1 - j, j);
      A.at(2 * KL + 1, 1) = A.at(2 * KL + 1, 1) - D.R(1, -1);
    }
    if (o.cfg.vel_bc == 1 || o.cfg.vel_bc == 3) {
      A.at(2 * KL + 1, N) = 1.0;
    } else {
      for (int j = N - KL; j <= N; ++j) A.at(2 * KL + 1 + N - j, j) = D.dr[1].at(KL + 1 + N - j, j);
      A.at(2 * KL + 1, N) = A.at(2 * KL + 1, N) - D.R(N, -1);
    }
    bad |= lu_find(A);
    if (bq) tim_mesh_flayer_Y(o, D, c1, c2, l, o.YTor[l]);
    else tim_mesh_vel_Y(o, D, c1, c2, l, o.YTor[l]);
  }
  for (int l = 1; l < L; ++l) {
    if (bq) tim_lumesh_flayer_X(o, D, c1, c2, l, o.XPol[l]);
    else tim_lumesh_vel_X(o, D, c1, c2, l, o.XPol[l]);
    LUBand& A = o.XPol[l];  // vel_bc_Pol (velocity.F90:207-254)
    if (o.cfg.vel_bc == 1 || o.cfg.vel_bc == 2) {
      for (int j = 1; j <= 1 + KL; ++j) A.at(2 * KL + 1 + 1 - j, j) = D.dr[1].at(KL + 1 + 1 - j, j);
    } else if (bq) {
      for (int j = 1; j <= 1 + KL; ++j) A.at(2 * KL + 1 + 1 - j, j) = D.dr[2].at(KL + 1 + 1 - j, j);
    } else {  // compressible part of the stress-free condition
      for (int j = 1; j <= 1 + KL; ++j)
        A.at(2 * KL + 1 + 1 - j, j) = D.dr[2].at(KL + 1 + 1 - j, j) + D.rho1[0] * D.dr[1].at(KL + 1 + 1 - j, j);
    }
    if (o.cfg.vel_bc == 1 || o.cfg.vel_bc == 3) {
      for (int j = N - KL; j <= N; ++j) A.at(2 * KL + 1 + N - j, j) = D.dr[1].at(KL + 1 + N - j, j);
    } else if (!bq) {
      for (int j = N - KL; j <= N; ++j)
        A.at(2 * KL + 1 + N - j, j) = D.dr[2].at(KL + 1 + N - j, j) + D.rho1[N - 1] * D.dr[1].at(KL + 1 + N - j, j);
    } else {
      for (int j = N - KL; j <= N; ++j) A.at(2 * KL + 1 + N - j, j) = D.dr[2].at(KL + 1 + N - j, j);
    }
    bad |= lu_find(A);
    if (bq) tim_mesh_flayer_Y(o, D, c1, c2, l, o.YPol[l]);
    else tim_mesh_vel_Y(o, D, c1, c2, l, o.YPol[l]);
  }
  c1 = 0.0; c2 = 1.0 / o.cfg.implicit;
  for (int l = 1; l < L; ++l) {
    if (bq) tim_lumesh_flayer_X(o, D, c1, c2, l, o.XGre[l]);
    else tim_lumesh_Gre_X(o, D, c1, c2, l, o.XGre[l]);
    o.XGre[l].at(2 * KL + 1, 1) = 1.0;  // vel_bc_Gre (velocity.F90:260-267)
    o.XGre[l].at(2 * KL + 1, N) = 1.0;
    bad |= lu_find(o.XGre[l]);
  }
  o.Gre.assign((size_t)N * 2 * L, 0.0);
  o.invG.assign((size_t)4 * L, 0.0);
  std::vector<double> pr(N), pi(N);
  for (int l = 1; l < L; ++l) {
    std::fill(pr.begin(), pr.end(), 0.0); std::fill(pi.begin(), pi.end(), 0.0);
    pr[0] = 1.0; pi[N - 1] = 1.0;
    for (double* b : {pr.data(), pi.data()})
      dgbtrs1(N, KL, KL, o.XGre[l].M.data(), 3 * KL + 1, o.XGre[l].ipiv.data(), b);
    pr[0] = 0; pr[N - 1] = 0; pi[0] = 0; pi[N - 1] = 0;  // tim_zerobc
    for (double* b : {pr.data(), pi.data()})
      dgbtrs1(N, KL, KL, o.XPol[l].M.data(), 3 * KL + 1, o.XPol[l].ipiv.data(), b);
    double* G = &o.Gre[(size_t)N * 2 * l];
    for (int n = 0; n < N; ++n) { G[n] = pr[n]; G[N + n] = pi[n]; }
    double* iG = &o.invG[(size_t)4 * l];  // invG(i,j) -> iG[(i-1) + 2(j-1)]
    iG[0] = G[0]; iG[2] = G[N]; iG[1] = G[N - 1]; iG[3] = G[N + N - 1];
    bad |= mat_invert(2, iG, 2);
  }
  // cod_matrices (codensity.F90:37-79), comp_matrices (composition.F90:31-54)
  for (int which = 0; which < 2; ++which) {
    std::vector<LUBand>& X = which == 0 ? o.XC : o.XComp;
    std::vector<Band>& Y = which == 0 ? o.YC : o.YComp;
    int bc = which == 0 ? o.cfg.cod_bc : o.cfg.comp_bc;
    double cc1 = which == 0 ? o.cfg.Pr / o.cfg.Pm : o.cfg.Sc / o.cfg.Pm;
    for (int l = 0; l < L; ++l) {
      tim_lumesh_X(o, D, cc1, 1.0, l, X[l]);
      LUBand& A = X[l];
      if (bc == 1 || bc == 2) A.at(2 * KL + 1, 1) = 1.0;
      else for (int j = 1; j <= 1 + KL; ++j) A.at(2 * KL + 1 + 1 - j, j) = D.dr[1].at(KL + 1 + 1 - j, j);
      if (bc == 1 || bc == 3) A.at(2 * KL + 1, N) = 1.0;
      else for (int j = N - KL; j <= N; ++j) A.at(2 * KL + 1 + N - j, j) = D.dr[1].at(KL + 1 + N - j, j);
      bad |= lu_find(A);
      tim_mesh_Y(o, D, cc1, 1.0, l, Y[l]);
    }
  }
  // mag_matrices (magnetic.F90:62-133); conducting inner core: the coupled operators
  // and tim_mesh_Y on the inner-core mesh (the Boussinesq equations)
  if (o.Nic > 1) {
    o.icYTor.assign(L, Band()); o.icYPol.assign(L, Band());
    for (int l = 1; l < L; ++l) {
      tim_iclumesh_X_cic(o, 1.0, 1.0, l, true, o.mXTor[l]);
      bad |= lu_find(o.mXTor[l]);
      tim_mesh_Y(o, D, 1.0, 1.0, l, o.mYTor[l]);
      tim_mesh_Y(o, o.ic, 1.0, 1.0, l, o.icYTor[l]);
    }
    for (int l = 1; l < L; ++l) {
      tim_iclumesh_X_cic(o, 1.0, 1.0, l, false, o.mXPol[l]);
      bad |= lu_find(o.mXPol[l]);
      tim_mesh_Y(o, D, 1.0, 1.0, l, o.mYPol[l]);
      tim_mesh_Y(o, o.ic, 1.0, 1.0, l, o.icYPol[l]);
    }
    return bad ? 1 : 0;
  }
  // insulating inner core (Ni = 1)
  for (int l = 1; l < L; ++l) {
    if (bq) tim_iclumesh_X(o, D, 1.0, 1.0, l, true, o.mXTor[l]);
    else tim_iclumesh_X_anel(o, D, 1.0, 1.0, l, true, o.mXTor[l]);
    o.mXTor[l].at(2 * KL + 1, 1) = 1.0;  // mag_bc_Tor (magnetic.F90:137-192)
    o.mXTor[l].at(2 * KL + 1, N) = 1.0;
    bad |= lu_find(o.mXTor[l]);
    if (bq) tim_mesh_Y(o, D, 1.0, 1.0, l, o.mYTor[l]);
    else tim_mesh_mag_Y(o, D, 1.0, 1.0, l, true, o.mYTor[l]);
  }
  for (int l = 1; l < L; ++l) {
    if (bq) tim_iclumesh_X(o, D, 1.0, 1.0, l, false, o.mXPol[l]);
    else tim_iclumesh_X_anel(o, D, 1.0, 1.0, l, false, o.mXPol[l]);
    LUBand& A = o.mXPol[l];  // mag_bc_Pol (magnetic.F90:198-282), Ni = 1, homogeneous
    for (int j = 1; j <= 1 + KL; ++j) A.at(2 * KL + 1 + 1 - j, j) = D.dr[1].at(KL + 1 + 1 - j, j);
    A.at(2 * KL + 1, 1) = A.at(2 * KL + 1, 1) - D.R(1, -1) * l;
    for (int j = N - KL; j <= N; ++j) A.at(2 * KL + 1 + N - j, j) = D.dr[1].at(KL + 1 + N - j, j);
    A.at(2 * KL + 1, N) = A.at(2 * KL + 1, N) + D.R(N, -1) * (l + 1);
    bad |= lu_find(A);
    if (bq) tim_mesh_Y(o, D, 1.0, 1.0, l, o.mYPol[l]);
    else tim_mesh_mag_Y(o, D, 1.0, 1.0, l, false, o.mYPol[l]);
  }
  return bad ? 1 : 0;
}

// ========================================================================================
// FFT row transforms (tra_s2p / tra_p2s serial branches, transform.fftw3.F90:280-466)
// ========================================================================================
// Y3: (Th, 0:2Hc-1) complex per shell/field -> X: (Th, 0:Ph-1)
void s2p_shell(const Oracle& o, const cplx* Y3, double* X, cplx* bufA, cplx* bufB, cplx* scr) {
  int Th = o.Th, Ph = o.Ph;
  for (int j = 0; j < Th; ++j) {
    // a2c_Y(j, 0:Ma): bins from the m-counter map, bins >= M zero
    for (int b = 0; b < Ph; ++b) bufA[b] = 0.0;
    for (int m = 0; m < 2 * o.Hc; ++m) {
      int mp = o.thm[m];
      if (mp < o.M) {
        cplx y = Y3[j + (size_t)Th * m];
        if (mp == 0) {
          bufA[0] = cplx(y.real(), 0.0);
        } else {
          bufA[mp] = y;
          bufA[Ph - mp] = std::conj(y);
        }
      }
    }
    o.fft.exec(bufA, bufB, +1, scr);
    for (int i = 0; i < Ph; ++i) X[j + (size_t)Th * i] = bufB[i].real();
  }
}
void p2s_shell(const Oracle& o, const double* X, cplx* Y3, cplx* bufA, cplx* bufB, cplx* scr) {
  int Th = o.Th, Ph = o.Ph;
  double scale = 1.0 / (double)Ph;
  for (int j = 0; j < Th; ++j) {
    for (int i = 0; i < Ph; ++i) bufA[i] = cplx(X[j + (size_t)Th * i] * scale, 0.0);
    o.fft.exec(bufA, bufB, -1, scr);
    bufB[0] = cplx(bufB[0].real(), 0.0);
    for (int m = 0; m < 2 * o.Hc; ++m) {
      int mp = o.thm[m];
      Y3[j + (size_t)Th * m] = bufB[mp];
    }
  }
}

struct Work {
  std::vector<cplx> a, b, scr;
  std::vector<cplx> Y[4];  // Y(Th2, 0:2Hc-1, 0:1)
  std::vector<cplx> Y3[3];  // (Th, 0:2Hc-1)
  void init(const Oracle& o) {
    a.resize(o.Ph); b.resize(o.Ph); scr.resize(o.Ph);
    for (auto& y : Y) y.resize((size_t)o.Th2 * 2 * o.Hc * 2);
    for (auto& y : Y3) y.resize((size_t)o.Th * 2 * o.Hc);
  }
};
inline size_t yidx(const Oracle& o, int j, int m, int s) { return (size_t)j + (size_t)o.Th2 * (m + (size_t)2 * o.Hc * s); }

// Y(:,m,0)+Y(:,m,1) on j <= Th2 ; Y(Th_:1:-1,:,0) - Y(Th_:1:-1,:,1) on j > Th2
void combine_ns(const Oracle& o, const std::vector<cplx>& Y, std::vector<cplx>& Y3) {
  int Th = o.Th, Th2 = o.Th2, Th_ = o.Th / 2;
  for (int m = 0; m < 2 * o.Hc; ++m) {
    for (int j = 0; j < Th2; ++j) Y3[j + (size_t)Th * m] = Y[yidx(o, j, m, 0)] + Y[yidx(o, j, m, 1)];
    for (int k = 0; k < Th - Th2; ++k) {
      int js = Th_ - 1 - k;  // Y(Th_:1:-1)
      Y3[Th2 + k + (size_t)Th * m] = Y[yidx(o, js, m, 0)] - Y[yidx(o, js, m, 1)];
    }
  }
}
// parity fold for analysis (transform.fftw3.F90:544-549)
void fold_ns(const Oracle& o, const cplx* Y3, std::vector<cplx>& Y) {
  int Th = o.Th, Th2 = o.Th2, Th_ = o.Th / 2 + 1;
  for (int m = 0; m < 2 * o.Hc; ++m) {
    for (int j = 0; j < Th2; ++j) {
      cplx a = Y3[j + (size_t)Th * m], b = Y3[(Th - 1 - j) + (size_t)Th * m];
      Y[yidx(o, j, m, 0)] = a + b;
      Y[yidx(o, j, m, 1)] = a - b;
    }
    if (Th2 == Th_) Y[yidx(o, Th2 - 1, m, 0)] = Y[yidx(o, Th2 - 1, m, 0)] * 0.5;
  }
}

// m-counter for each nh (the _loop_sumth m)
std::vector<int> mcount(const Oracle& o) {
  std::vector<int> mc(o.H);
  int m = -1, m_ = -1;
  for (int nh = 0; nh < o.H; ++nh) {
    int m__ = m_;
    m_ = o.hm[nh];
    if (m_ != m__) ++m;
    mc[nh] = m;
  }
  return mc;
}

// ---- tra_spec2phys (transform.fftw3.F90:472-520) ---------------------------------------
void tra_spec2phys(const Oracle& o, const Spec& s, Phys& p) {
  std::vector<int> mc = mcount(o);
  p.assign((size_t)o.Th * o.Ph * o.N, 0.0);
#pragma omp parallel
  {
    Work w; w.init(o);
#pragma omp for schedule(static)
    for (int n = 0; n < o.N; ++n) {
      std::fill(w.Y[0].begin(), w.Y[0].end(), cplx(0, 0));
      for (int nh = 0; nh < o.H; ++nh) {
        cplx c(s.re[nh + (size_t)o.H * n], s.im[nh + (size_t)o.H * n]);
        const double* P = &o.P[(size_t)o.Th2 * nh];
        cplx* Y = &w.Y[0][yidx(o, 0, mc[nh], o.hs[nh])];
        for (int j = 0; j < o.Th2; ++j) Y[j] = Y[j] + c * P[j];
      }
      combine_ns(o, w.Y[0], w.Y3[0]);
      s2p_shell(o, w.Y3[0].data(), &p[(size_t)o.Th * o.Ph * n], w.a.data(), w.b.data(), w.scr.data());
    }
  }
}

// ---- tra_phys2spec (transform.fftw3.F90:527-602) ---------------------------------------
void tra_phys2spec(const Oracle& o, const Phys& p, Spec& s) {
  std::vector<int> mc = mcount(o);
  s.init(o.N, o.H);
#pragma omp parallel
  {
    Work w; w.init(o);
#pragma omp for schedule(static)
    for (int n = 0; n < o.N; ++n) {
      p2s_shell(o, &p[(size_t)o.Th * o.Ph * n], w.Y3[0].data(), w.a.data(), w.b.data(), w.scr.data());
      fold_ns(o, w.Y3[0].data(), w.Y[0]);
      for (int nh = 0; nh < o.H; ++nh) {
        const cplx* Y = &w.Y[0][yidx(o, 0, mc[nh], o.hs[nh])];
        const double* W = &o.gwP[(size_t)o.Th2 * nh];
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < o.Th2; ++j) { sr = sr + Y[j].real() * W[j]; si = si + Y[j].imag() * W[j]; }
        s.re[nh + (size_t)o.H * n] = sr;
        s.im[nh + (size_t)o.H * n] = (o.hm[nh] == 0) ? 0.0 : si;
      }
    }
  }
}

// ---- tra_qst2rtp (transform.fftw3.F90:719-818) -----------------------------------------
void tra_qst2rtp(const Oracle& o, const Spec& q, const Spec& s, const Spec& t, Phys& r, Phys& th, Phys& ph) {
  std::vector<int> mc = mcount(o);
  size_t psz = (size_t)o.Th * o.Ph * o.N;
  r.assign(psz, 0.0); th.assign(psz, 0.0); ph.assign(psz, 0.0);
#pragma omp parallel
  {
    Work w; w.init(o);
#pragma omp for schedule(static)
    for (int n = 0; n < o.N; ++n) {
      for (int k = 0; k < 3; ++k) std::fill(w.Y[k].begin(), w.Y[k].end(), cplx(0, 0));
      for (int nh = 0; nh < o.H; ++nh) {
        size_t i = nh + (size_t)o.H * n;
        int m = mc[nh], sp = o.hs[nh];
        cplx c1(q.re[i], q.im[i]);
        const double* P = &o.P[(size_t)o.Th2 * nh];
        cplx* Y1 = &w.Y[0][yidx(o, 0, m, sp)];
        for (int j = 0; j < o.Th2; ++j) Y1[j] = Y1[j] + c1 * P[j];
      }
      for (int nh = 0; nh < o.H; ++nh) {
        size_t i = nh + (size_t)o.H * n;
        int m = mc[nh], sp = o.hs[nh];
        cplx c1(s.re[i], s.im[i]), c2(t.im[i], -t.re[i]), c3(-s.im[i], s.re[i]), c4(t.re[i], t.im[i]);
        const double* A1 = &o.llP_[(size_t)o.Th2 * nh];
        const double* A2 = &o.llsin1mP[(size_t)o.Th2 * nh];
        cplx* Y2a = &w.Y[1][yidx(o, 0, m, 1 - sp)];
        cplx* Y2b = &w.Y[1][yidx(o, 0, m, sp)];
        cplx* Y3a = &w.Y[2][yidx(o, 0, m, sp)];
        cplx* Y3b = &w.Y[2][yidx(o, 0, m, 1 - sp)];
        for (int j = 0; j < o.Th2; ++j) {
          Y2a[j] = Y2a[j] + c1 * A1[j];
          Y2b[j] = Y2b[j] + c2 * A2[j];
          Y3a[j] = Y3a[j] + c3 * A2[j];
          Y3b[j] = Y3b[j] + c4 * A1[j];
        }
      }
      Phys* outs[3] = {&r, &th, &ph};
      for (int k = 0; k < 3; ++k) {
        combine_ns(o, w.Y[k], w.Y3[k]);
        s2p_shell(o, w.Y3[k].data(), &(*outs[k])[(size_t)o.Th * o.Ph * n], w.a.data(), w.b.data(), w.scr.data());
      }
    }
  }
}

// ---- tra_qst2rtp_vel (transform.fftw3.F90:611-714), anelastic -----------------------------
// outs: r, th, ph, dur, qv1, dutr, dupr, qv2
void tra_qst2rtp_vel(const Oracle& o, const Spec& q, const Spec& s, const Spec& t, const Spec& qr, const Spec& sr,
                     const Spec& tr, Phys* outs[8]) {
  std::vector<int> mc = mcount(o);
  size_t psz = (size_t)o.Th * o.Ph * o.N;
  for (int k = 0; k < 8; ++k) outs[k]->assign(psz, 0.0);
#pragma omp parallel
  {
    Work w; w.init(o);
    std::vector<cplx> Y3b((size_t)o.Th * 2 * o.Hc);
    auto emit = [&](int k, const std::vector<cplx>& Y, int n) {
      combine_ns(o, Y, Y3b);
      s2p_shell(o, Y3b.data(), &(*outs[k])[(size_t)o.Th * o.Ph * n], w.a.data(), w.b.data(), w.scr.data());
    };
#pragma omp for schedule(static)
    for (int n = 0; n < o.N; ++n) {
      // Ar = q, dur = qr
      for (int k = 0; k < 2; ++k) std::fill(w.Y[k].begin(), w.Y[k].end(), cplx(0, 0));
      for (int nh = 0; nh < o.H; ++nh) {
        size_t i = nh + (size_t)o.H * n;
        int m = mc[nh], sp = o.hs[nh];
        cplx c1(q.re[i], q.im[i]), c2(qr.re[i], qr.im[i]);
        const double* P = &o.P[(size_t)o.Th2 * nh];
        cplx* Y1 = &w.Y[0][yidx(o, 0, m, sp)];
        cplx* Y2 = &w.Y[1][yidx(o, 0, m, sp)];
        for (int j = 0; j < o.Th2; ++j) { Y1[j] = Y1[j] + c1 * P[j]; Y2[j] = Y2[j] + c2 * P[j]; }
      }
      emit(0, w.Y[0], n);
      emit(3, w.Y[1], n);
      // At = s dth - t/sin dph, and the same of (sr, tr)
      for (int k = 0; k < 2; ++k) std::fill(w.Y[k].begin(), w.Y[k].end(), cplx(0, 0));
      for (int nh = 0; nh < o.H; ++nh) {
        size_t i = nh + (size_t)o.H * n;
        int m = mc[nh], sp = o.hs[nh];
        cplx c1(s.re[i], s.im[i]), c2(t.im[i], -t.re[i]), c3(sr.re[i], sr.im[i]), c4(tr.im[i], -tr.re[i]);
        const double* A1 = &o.llP_[(size_t)o.Th2 * nh];
        const double* A2 = &o.llsin1mP[(size_t)o.Th2 * nh];
        cplx* Y1o = &w.Y[0][yidx(o, 0, m, 1 - sp)];
        cplx* Y1s = &w.Y[0][yidx(o, 0, m, sp)];
        cplx* Y2o = &w.Y[1][yidx(o, 0, m, 1 - sp)];
        cplx* Y2s = &w.Y[1][yidx(o, 0, m, sp)];
        for (int j = 0; j < o.Th2; ++j) {
          Y1o[j] = Y1o[j] + c1 * A1[j];
          Y1s[j] = Y1s[j] + c2 * A2[j];
          Y2o[j] = Y2o[j] + c3 * A1[j];
          Y2s[j] = Y2s[j] + c4 * A2[j];
        }
      }
      emit(1, w.Y[0], n);
      emit(5, w.Y[1], n);
      // Aph = s/sin dph + t dth, the same of (sr, tr), and the qva / qvb sums
      for (int k = 0; k < 4; ++k) std::fill(w.Y[k].begin(), w.Y[k].end(), cplx(0, 0));
      double rinv = o.oc.R(n + 1, -1);
      for (int nh = 0; nh < o.H; ++nh) {
        size_t i = nh + (size_t)o.H * n;
        int m = mc[nh], sp = o.hs[nh];
        cplx c1(-s.im[i], s.re[i]), c2(t.re[i], t.im[i]), c3(-sr.im[i], sr.re[i]), c4(tr.re[i], tr.im[i]);
        cplx c5(-s.re[i] * rinv, -s.im[i] * rinv), c6(t.im[i] * rinv, -t.re[i] * rinv);
        cplx c7(t.re[i] * rinv, t.im[i] * rinv), c8(s.im[i] * rinv, -s.re[i] * rinv);
        const double* A1 = &o.llP_[(size_t)o.Th2 * nh];
        const double* A2 = &o.llsin1mP[(size_t)o.Th2 * nh];
        const double* QA = &o.qva[(size_t)o.Th2 * nh];
        const double* QB = &o.qvb[(size_t)o.Th2 * nh];
        cplx* Y1s = &w.Y[0][yidx(o, 0, m, sp)];
        cplx* Y1o = &w.Y[0][yidx(o, 0, m, 1 - sp)];
        cplx* Y2s = &w.Y[1][yidx(o, 0, m, sp)];
        cplx* Y2o = &w.Y[1][yidx(o, 0, m, 1 - sp)];
        cplx* Y3s = &w.Y[2][yidx(o, 0, m, sp)];
        cplx* Y3o = &w.Y[2][yidx(o, 0, m, 1 - sp)];
        cplx* Y4s = &w.Y[3][yidx(o, 0, m, sp)];
        cplx* Y4o = &w.Y[3][yidx(o, 0, m, 1 - sp)];
        for (int j = 0; j < o.Th2; ++j) {
          Y1s[j] = Y1s[j] + c1 * A2[j];
          Y1o[j] = Y1o[j] + c2 * A1[j];
          Y2s[j] = Y2s[j] + c3 * A2[j];
          Y2o[j] = Y2o[j] + c4 * A1[j];
          Y3s[j] = Y3s[j] + c5 * QA[j];
          Y3o[j] = Y3o[j] + c6 * QB[j];
          Y4s[j] = Y4s[j] + c7 * QA[j];
          Y4o[j] = Y4o[j] + c8 * QB[j];
        }
      }
      emit(2, w.Y[0], n);
      emit(6, w.Y[1], n);
      emit(4, w.Y[2], n);
      emit(7, w.Y[3], n);
    }
  }
}

// ---- tra_rtp2qst (transform.fftw3.F90:825-949) -----------------------------------------
void tra_rtp2qst(const Oracle& o, const Phys& r, const Phys& th, const Phys& ph, Spec& q, Spec& s, Spec& t) {
  std::vector<int> mc = mcount(o);
  q.init(o.N, o.H); s.init(o.N, o.H); t.init(o.N, o.H);
#pragma omp parallel
  {
    Work w; w.init(o);
#pragma omp for schedule(static)
    for (int n = 0; n < o.N; ++n) {
      const Phys* ins[3] = {&r, &th, &ph};
      for (int k = 0; k < 3; ++k) {
        p2s_shell(o, &(*ins[k])[(size_t)o.Th * o.Ph * n], w.Y3[k].data(), w.a.data(), w.b.data(), w.scr.data());
        fold_ns(o, w.Y3[k].data(), w.Y[k]);
      }
      for (int nh = 0; nh < o.H; ++nh) {
        size_t i = nh + (size_t)o.H * n;
        int m = mc[nh], sp = o.hs[nh];
        const double* gP = &o.gwP[(size_t)o.Th2 * nh];
        const double* gA1 = &o.gwllP_[(size_t)o.Th2 * nh];
        const double* gA2 = &o.gwllsin1mP[(size_t)o.Th2 * nh];
        const cplx* Y1 = &w.Y[0][yidx(o, 0, m, sp)];
        double a = 0, b = 0;
        for (int j = 0; j < o.Th2; ++j) { a = a + Y1[j].real() * gP[j]; b = b + Y1[j].imag() * gP[j]; }
        q.re[i] = a; q.im[i] = b;   // q%Im of m=0 is not zeroed (the quirk at :869)
        const cplx* Y2o = &w.Y[1][yidx(o, 0, m, 1 - sp)];
        const cplx* Y2s = &w.Y[1][yidx(o, 0, m, sp)];
        const cplx* Y3s = &w.Y[2][yidx(o, 0, m, sp)];
        const cplx* Y3o = &w.Y[2][yidx(o, 0, m, 1 - sp)];
        double sr = 0, si = 0, tr = 0, ti = 0, x;
        for (int j = 0; j < o.Th2; ++j) { sr = sr + Y2o[j].real() * gA1[j]; si = si + Y2o[j].imag() * gA1[j]; }
        x = 0; for (int j = 0; j < o.Th2; ++j) x = x + Y2s[j].imag() * gA2[j];
        tr = -x;
        x = 0; for (int j = 0; j < o.Th2; ++j) x = x + Y2s[j].real() * gA2[j];
        ti = x;
        x = 0; for (int j = 0; j < o.Th2; ++j) x = x + Y3s[j].imag() * gA2[j];
        sr = sr + x;
        x = 0; for (int j = 0; j < o.Th2; ++j) x = x + Y3s[j].real() * gA2[j];
        si = si - x;
        if (o.hm[nh] == 0) si = 0.0;
        x = 0; for (int j = 0; j < o.Th2; ++j) x = x + Y3o[j].real() * gA1[j];
        tr = tr + x;
        x = 0; for (int j = 0; j < o.Th2; ++j) x = x + Y3o[j].imag() * gA1[j];
        ti = ti + x;
        if (o.hm[nh] == 0) ti = 0.0;
        s.re[i] = sr; s.im[i] = si; t.re[i] = tr; t.im[i] = ti;
      }
    }
  }
}

// ---- tra_grad (transform.fftw3.F90:955-1000) -------------------------------------------
void tra_grad(const Oracle& o, const Spec& s, Phys& tp, Phys& pp) {
  std::vector<int> mc = mcount(o);
  size_t psz = (size_t)o.Th * o.Ph * o.N;
  tp.assign(psz, 0.0); pp.assign(psz, 0.0);
#pragma omp parallel
  {
    Work w; w.init(o);
#pragma omp for schedule(static)
    for (int n = 0; n < o.N; ++n) {
      double r1 = o.oc.R(n + 1, -1);
      std::fill(w.Y[0].begin(), w.Y[0].end(), cplx(0, 0));
      std::fill(w.Y[1].begin(), w.Y[1].end(), cplx(0, 0));
      for (int nh = 0; nh < o.H; ++nh) {
        size_t i = nh + (size_t)o.H * n;
        cplx c(s.re[i], s.im[i]);
        c = c * r1;
        const double* A = &o.P_[(size_t)o.Th2 * nh];
        cplx* Y = &w.Y[0][yidx(o, 0, mc[nh], 1 - o.hs[nh])];
        for (int j = 0; j < o.Th2; ++j) Y[j] = Y[j] + c * A[j];
      }
      for (int nh = 0; nh < o.H; ++nh) {
        size_t i = nh + (size_t)o.H * n;
        cplx c(-s.im[i], s.re[i]);
        c = c * r1;
        const double* A = &o.sin1mP[(size_t)o.Th2 * nh];
        cplx* Y = &w.Y[1][yidx(o, 0, mc[nh], o.hs[nh])];
        for (int j = 0; j < o.Th2; ++j) Y[j] = Y[j] + c * A[j];
      }
      combine_ns(o, w.Y[0], w.Y3[0]);
      combine_ns(o, w.Y[1], w.Y3[1]);
      s2p_shell(o, w.Y3[0].data(), &tp[(size_t)o.Th * o.Ph * n], w.a.data(), w.b.data(), w.scr.data());
      s2p_shell(o, w.Y3[1].data(), &pp[(size_t)o.Th * o.Ph * n], w.a.data(), w.b.data(), w.scr.data());
    }
  }
}

// ---- tra_dth (transform.fftw3.F90:1006-1031) -------------------------------------------
void tra_dth(const Oracle& o, const Spec& s, Phys& pp) {
  std::vector<int> mc = mcount(o);
  pp.assign((size_t)o.Th * o.Ph * o.N, 0.0);
#pragma omp parallel
  {
    Work w; w.init(o);
#pragma omp for schedule(static)
    for (int n = 0; n < o.N; ++n) {
      std::fill(w.Y[0].begin(), w.Y[0].end(), cplx(0, 0));
      for (int nh = 0; nh < o.H; ++nh) {
        size_t i = nh + (size_t)o.H * n;
        cplx c(s.re[i], s.im[i]);
        const double* A = &o.P_[(size_t)o.Th2 * nh];
        cplx* Y = &w.Y[0][yidx(o, 0, mc[nh], 1 - o.hs[nh])];
        for (int j = 0; j < o.Th2; ++j) Y[j] = Y[j] + c * A[j];
      }
      combine_ns(o, w.Y[0], w.Y3[0]);
      s2p_shell(o, w.Y3[0].data(), &pp[(size_t)o.Th * o.Ph * n], w.a.data(), w.b.data(), w.scr.data());
    }
  }
}

// ========================================================================================
// coll algebra (variables.F90:246-829)
// ========================================================================================
void coll2spec(const Oracle& o, const Coll& c, Spec& s) {
  s.init(o.N, o.H);
  for (int nh = 0; nh < o.H; ++nh)
    for (int n = 0; n < o.N; ++n) {
      s.re[nh + (size_t)o.H * n] = c.re[n + (size_t)o.N * nh];
      s.im[nh + (size_t)o.H * n] = c.im[n + (size_t)o.N * nh];
    }
}
void spec2coll(const Oracle& o, const Spec& s, Coll& c) {
  c.init(o.N, o.H);
  for (int nh = 0; nh < o.H; ++nh)
    for (int n = 0; n < o.N; ++n) {
      c.re[n + (size_t)o.N * nh] = s.re[nh + (size_t)o.H * n];
      c.im[n + (size_t)o.N * nh] = s.im[nh + (size_t)o.H * n];
    }
}
// var_coll_meshmult (variables.F90:476-505)
void meshmult_n(const Oracle& o, int N, const Band& A, const Coll& in, Coll& out);
void meshmult(const Oracle& o, const Band& A, const Coll& in, Coll& out) { meshmult_n(o, o.N, A, in, out); }
void meshmult_n(const Oracle& o, int N, const Band& A, const Coll& in, Coll& out) {
  int KL = o.KL;
  Coll tmp; tmp.init(N, o.H);
  for (int nh = 0; nh < o.H; ++nh) {
    double* re = &tmp.re[(size_t)N * nh];
    double* im = &tmp.im[(size_t)N * nh];
    const double* ir = &in.re[(size_t)N * nh];
    const double* ii = &in.im[(size_t)N * nh];
    for (int j = 1; j <= N; ++j) {
      int l = std::max(1, j - KL), r = std::min(j + KL, N);
      for (int n = l; n <= r; ++n) {
        re[n - 1] = re[n - 1] + A.at(KL + 1 + n - j, j) * ir[j - 1];
        im[n - 1] = im[n - 1] + A.at(KL + 1 + n - j, j) * ii[j - 1];
      }
    }
  }
  out = std::move(tmp);
}
// var_coll_TorPol2qst_mag (variables.F90:565-605); with the Boussinesq zero rho the
// compressible var_coll_TorPol2qst (:511-556) is the same arithmetic up to the +0 of xi.
void torpol2qst_d(const Oracle& o, const RDom& D, const Coll& Tor, const Coll& Pol, Coll& q, Coll& s, Coll& t,
                  bool comp);
void torpol2qst(const Oracle& o, const Coll& Tor, const Coll& Pol, Coll& q, Coll& s, Coll& t, bool comp) {
  torpol2qst_d(o, o.oc, Tor, Pol, q, s, t, comp);
}
// the same on a radial domain D (the inner core's mesh for its energies)
void torpol2qst_d(const Oracle& o, const RDom& D, const Coll& Tor, const Coll& Pol, Coll& q, Coll& s, Coll& t,
                  bool comp) {
  int N = D.N;
  q.init(N, o.H); t.init(N, o.H);
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh];
    for (int n = 1; n <= N; ++n) {
      size_t i = (n - 1) + (size_t)N * nh;
      double a = o.ad_ll1[l] * D.R(n, -1);
      q.re[i] = Pol.re[i] * a;
      q.im[i] = Pol.im[i] * a;
    }
  }
  meshmult_n(o, N, comp ? D.compr1dr : D.r1dr, Pol, s);
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh];
    for (int n = 0; n < N; ++n) {
      size_t i = n + (size_t)N * nh;
      s.re[i] = s.re[i] * o.ad_rtll1[l];
      s.im[i] = s.im[i] * o.ad_rtll1[l];
      t.re[i] = -Tor.re[i] * o.ad_rtll1[l];
      t.im[i] = -Tor.im[i] * o.ad_rtll1[l];
    }
  }
}
// var_coll_TorPol2qstderiv (variables.F90:610-660): q, s (compressible), t and their
// radial derivatives dr(1) q, dr(1) s, dr(1) t
void torpol2qstderiv(const Oracle& o, const Coll& Tor, const Coll& Pol, Coll& q, Coll& s, Coll& t, Coll& qr,
                     Coll& sr, Coll& tr) {
  torpol2qst(o, Tor, Pol, q, s, t, true);
  meshmult(o, o.oc.dr[1], q, qr);
  meshmult(o, o.oc.dr[1], s, sr);
  meshmult(o, o.oc.dr[1], t, tr);
}
// var_coll_qstcurl (variables.F90:713-754)
void qstcurl_d(const Oracle& o, const RDom& D, const Coll& q, const Coll& s, const Coll& t, Coll& oq, Coll& os,
               Coll& ot);
void qstcurl(const Oracle& o, const Coll& q, const Coll& s, const Coll& t, Coll& oq, Coll& os, Coll& ot) {
  qstcurl_d(o, o.oc, q, s, t, oq, os, ot);
}
void qstcurl_d(const Oracle& o, const RDom& D, const Coll& q, const Coll& s, const Coll& t, Coll& oq, Coll& os,
               Coll& ot) {
  int N = D.N;
  Coll tt = t;
  Coll nt; meshmult_n(o, N, D.r1dr, s, nt);
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh];
    for (int n = 1; n <= N; ++n) {
      size_t i = (n - 1) + (size_t)N * nh;
      double a = o.ad_rtll1[l] * D.R(n, -1);
      nt.re[i] = nt.re[i] - a * q.re[i];
      nt.im[i] = nt.im[i] - a * q.im[i];
    }
  }
  Coll ns; meshmult_n(o, N, D.r1dr, tt, ns);
  for (size_t i = 0; i < ns.re.size(); ++i) { ns.re[i] = -ns.re[i]; ns.im[i] = -ns.im[i]; }
  Coll nq; nq.init(N, o.H);
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh];
    for (int n = 1; n <= N; ++n) {
      size_t i = (n - 1) + (size_t)N * nh;
      double a = -o.ad_rtll1[l] * D.R(n, -1);
      nq.re[i] = tt.re[i] * a;
      nq.im[i] = tt.im[i] * a;
    }
  }
  oq = std::move(nq); os = std::move(ns); ot = std::move(nt);
}
void qstllcurlr(const Oracle& o, const Coll& t, Coll& r) {
  r.init(o.N, o.H);
  for (int nh = 0; nh < o.H; ++nh)
    for (int n = 0; n < o.N; ++n) {
      size_t i = n + (size_t)o.N * nh;
      r.re[i] = -t.re[i] * o.ad_rtll11[o.hl[nh]];
      r.im[i] = -t.im[i] * o.ad_rtll11[o.hl[nh]];
    }
}
void qstllcurlcurlr(const Oracle& o, const Coll& q, const Coll& s, Coll& r) {
  meshmult(o, o.oc.r1dr, s, r);
  for (int nh = 0; nh < o.H; ++nh)
    for (int n = 1; n <= o.N; ++n) {
      size_t i = (n - 1) + (size_t)o.N * nh;
      double w = o.ad_rtll11[o.hl[nh]];
      r.re[i] = r.re[i] * w;
      r.re[i] = q.re[i] * o.oc.R(n, -1) - r.re[i];
      r.im[i] = r.im[i] * w;
      r.im[i] = q.im[i] * o.oc.R(n, -1) - r.im[i];
    }
}

// ========================================================================================
// Transforms of the fields (velocity.F90:310-350, codensity.F90:195-213,
// magnetic.F90:336-360) and nonlinear terms (nonlinear.F90:28-473)
// ========================================================================================
void vec_transform(Oracle& o, const Coll& Tor, const Coll& Pol, Phys& r, Phys& t, Phys& p, Phys& cr, Phys& ct, Phys& cp) {
  Coll q, s, tt;
  torpol2qst(o, Tor, Pol, q, s, tt, false);
  Spec sq, ss, st;
  coll2spec(o, q, sq); coll2spec(o, s, ss); coll2spec(o, tt, st);
  tra_qst2rtp(o, sq, ss, st, r, t, p);
  qstcurl(o, q, s, tt, q, s, tt);
  coll2spec(o, q, sq); coll2spec(o, s, ss); coll2spec(o, tt, st);
  tra_qst2rtp(o, sq, ss, st, cr, ct, cp);
}
// vel_transform, anelastic branch (velocity.F90:333-347)
void vel_transform_anel(Oracle& o) {
  Coll q, s, tt, qr, sr, tr;
  torpol2qstderiv(o, o.vTor, o.vPol, q, s, tt, qr, sr, tr);
  Spec sq, ss, st, sqr, ssr, str;
  coll2spec(o, q, sq); coll2spec(o, s, ss); coll2spec(o, tt, st);
  coll2spec(o, qr, sqr); coll2spec(o, sr, ssr); coll2spec(o, tr, str);
  Phys* outs[8] = {&o.vel_r, &o.vel_t, &o.vel_p, &o.vel_dur, &o.vel_qv1, &o.vel_dutr, &o.vel_dupr, &o.vel_qv2};
  tra_qst2rtp_vel(o, sq, ss, st, sqr, ssr, str, outs);
  qstcurl(o, q, s, tt, q, s, tt);
  coll2spec(o, q, sq); coll2spec(o, s, ss); coll2spec(o, tt, st);
  tra_qst2rtp(o, sq, ss, st, o.vel_cr, o.vel_ct, o.vel_cp);
}
// vel_angmomclr (velocity.F90:475-574): with stress-free walls (i_vel_bc = 4) remove the
// rigid rotation carried by the l = 1, m <= 1 toroidal modes
void vel_angmomclr(Oracle& o) {
  if (o.cfg.vel_bc != 4) return;
  const int N = o.N;
  const bool bq = o.cfg.boussinesq != 0;
  const std::vector<double>& wt = bq ? o.oc.intr2dr : o.oc.intr2dr_comp;
  const double w = 8.0 / 3.0 * d_PI;
  auto dot = [&](const std::vector<double>& f) { double a = 0; for (int n = 0; n < N; ++n) a = a + f[n] * wt[n]; return a; };
  std::vector<double> f1(N), f2(N);
  for (int n = 0; n < N; ++n) f2[n] = bq ? o.oc.R(n + 1, 2) : o.oc.R(n + 1, 1) * o.oc.R(n + 1, 1);
  double omz = 0, omx = 0, omy = 0;
  int nz = -1, nx = -1;
  for (int nh = 0; nh < o.H; ++nh) {
    if (o.hl[nh] != 1 || o.hm[nh] > 1) continue;
    double* re = &o.vTor.re[(size_t)N * nh];
    double* im = &o.vTor.im[(size_t)N * nh];
    if (o.hm[nh] == 0) {
      for (int n = 0; n < N; ++n) f1[n] = re[n] * o.oc.R(n + 1, 1);
      double Lz = w * dot(f1), Lz2 = w * dot(f2);
      omz = Lz / Lz2;
      nz = nh;
    } else {
      for (int n = 0; n < N; ++n) f1[n] = re[n] * o.oc.R(n + 1, 1);
      double Lx = 2.0 * w * dot(f1), Lx2 = 2.0 * w * dot(f2);
      for (int n = 0; n < N; ++n) f1[n] = im[n] * o.oc.R(n + 1, 1);
      double Ly = -2.0 * w * dot(f1), Ly2 = -2.0 * w * dot(f2);
      omx = Lx / Lx2;
      omy = Ly / Ly2;
      nx = nh;
    }
  }
  if (nz >= 0)
    for (int n = 0; n < N; ++n) o.vTor.re[(size_t)N * nz + n] = o.vTor.re[(size_t)N * nz + n] - omz * o.oc.R(n + 1, 1);
  if (nx >= 0)
    for (int n = 0; n < N; ++n) {
      o.vTor.re[(size_t)N * nx + n] = o.vTor.re[(size_t)N * nx + n] - omx * o.oc.R(n + 1, 1);
      o.vTor.im[(size_t)N * nx + n] = o.vTor.im[(size_t)N * nx + n] - omy * o.oc.R(n + 1, 1);
    }
}
void scal_transform(Oracle& o, const Coll& C, Phys& gr, Phys& gt, Phys& gp) {
  Coll cC; meshmult(o, o.oc.dr[1], C, cC);
  Spec sC, sC_;
  coll2spec(o, C, sC); coll2spec(o, cC, sC_);
  tra_spec2phys(o, sC_, gr);
  tra_grad(o, sC, gt, gp);
}

void non_rotation(Oracle& o);
void evaluate(Oracle& o) {
  size_t psz = (size_t)o.Th * o.Ph * o.N;
  int Th = o.Th, Ph = o.Ph;
  const bool bq = o.cfg.boussinesq != 0;
  // transforms (main.F90:101-107)
  vel_angmomclr(o);
  if (bq) vec_transform(o, o.vTor, o.vPol, o.vel_r, o.vel_t, o.vel_p, o.vel_cr, o.vel_ct, o.vel_cp);
  else vel_transform_anel(o);
  scal_transform(o, o.codC, o.cod_gr, o.cod_gt, o.cod_gp);
  if (o.cfg.comp_tstep) scal_transform(o, o.compC, o.comp_gr, o.comp_gt, o.comp_gp);
  vec_transform(o, o.bTor, o.bPol, o.mag_r, o.mag_t, o.mag_p, o.mag_cr, o.mag_ct, o.mag_cp);
  if (o.cfg.rot_tstep) non_rotation(o);
  Phys r(psz), th(psz), ph(psz);
  // ---- non_velocity (nonlinear.F90:28-199)
  {
    double d_Cor = 2.0 * o.cfg.Pm / o.cfg.E;
    const double Pm = o.cfg.Pm;
#pragma omp parallel for schedule(static)
    for (int n = 0; n < o.N; ++n) {
      const double Cmag = bq ? 2 * o.cfg.Pm / o.cfg.E : o.cfg.Pm / (o.cfg.E * o.oc.rho0[n]);
      const double xi0 = o.oc.rho1[n], xi1 = o.oc.rho2[n], rm1 = o.oc.R(n + 1, -1);
      for (int m = 0; m < Ph; ++m)
        for (int j = 0; j < Th; ++j) {
          size_t i = j + (size_t)Th * (m + (size_t)Ph * n);
          double vr = o.vel_r[i], vt = o.vel_t[i], vp = o.vel_p[i];
          double wr = o.vel_cr[i], wt = o.vel_ct[i], wp = o.vel_cp[i];
          double a = vt * wp - vp * wt;
          double b = vp * wr - vr * wp;
          double c = vr * wt - vt * wr;
          if (!bq) {  // compressible part of the viscous force (nonlinear.F90:93-110)
            double f = -(2.0 * xi0 * rm1) - xi1;
            f = f - (xi0 * xi0) / 3.0;
            a = a + Pm * vr * f;
            double d1 = 2.0 * xi0 * rm1 + xi1;
            d1 = d1 + xi0 * xi0;
            b = b - Pm * (xi0 * wp + d1 * vt);
            c = c + Pm * (xi0 * wt - d1 * vp);
          }
          a = a + d_Cor * o.sn[j] * vp;
          b = b + d_Cor * o.gp[j] * vp;
          c = c - d_Cor * (o.gp[j] * vt + o.sn[j] * vr);
          a = a + Cmag * (o.mag_ct[i] * o.mag_p[i] - o.mag_cp[i] * o.mag_t[i]);
          b = b + Cmag * (o.mag_cp[i] * o.mag_r[i] - o.mag_cr[i] * o.mag_p[i]);
          c = c + Cmag * (o.mag_cr[i] * o.mag_t[i] - o.mag_ct[i] * o.mag_r[i]);
          r[i] = a; th[i] = b; ph[i] = c;
        }
    }
    Spec sq, ss, st;
    tra_rtp2qst(o, r, th, ph, sq, ss, st);
    Coll cq, cs, ct;
    spec2coll(o, sq, cq); spec2coll(o, ss, cs); spec2coll(o, st, ct);
    for (int nh = 0; nh < o.H; ++nh)
      for (int n = 1; n <= o.N; ++n) {
        double d2 = bq ? o.cfg.Ra * o.oc.R(n, 1) * (o.cfg.Pm * o.cfg.Pm) / o.cfg.Pr
                       : -(o.cfg.Ra * o.oc.temp1[n - 1] * (o.cfg.Pm * o.cfg.Pm) / o.cfg.Pr);
        size_t i = (n - 1) + (size_t)o.N * nh;
        cq.re[i] = cq.re[i] + d2 * o.codC.re[i];
        cq.im[i] = cq.im[i] + d2 * o.codC.im[i];
      }
    for (int nh = 0; nh < o.H; ++nh)
      for (int n = 1; n <= o.N; ++n) {
        double d2 = bq ? o.cfg.Ra_comp * o.oc.R(n, 1) * (o.cfg.Pm * o.cfg.Pm) / o.cfg.Sc
                       : -(o.cfg.Ra_comp * o.oc.temp1[n - 1] * (o.cfg.Pm * o.cfg.Pm) / o.cfg.Sc);
        size_t i = (n - 1) + (size_t)o.N * nh;
        cq.re[i] = cq.re[i] + d2 * o.compC.re[i];
        cq.im[i] = cq.im[i] + d2 * o.compC.im[i];
      }
    qstllcurlr(o, ct, o.vNTor);
    qstllcurlcurlr(o, cq, cs, o.vNPol);
    for (int n = 0; n < o.N; ++n) { o.vNTor.re[n] = 0; o.vNTor.im[n] = 0; o.vNPol.re[n] = 0; o.vNPol.im[n] = 0; }
  }
  // ---- non_codensity / non_composition (nonlinear.F90:205-357); composition keeps the
  // Boussinesq form in both cases, the anelastic codensity (entropy) adds the reference
  // temperature gradient term and the viscous + ohmic dissipation (nonlinear.F90:239-266)
  for (int which = 0; which < (o.cfg.comp_tstep ? 2 : 1); ++which) {
    double d_qm1 = which == 0 ? o.cfg.Pr / o.cfg.Pm : o.cfg.Sc / o.cfg.Pm;
    const Phys& gr = which == 0 ? o.cod_gr : o.comp_gr;
    const Phys& gt = which == 0 ? o.cod_gt : o.comp_gt;
    const Phys& gq = which == 0 ? o.cod_gp : o.comp_gp;
    if (bq || which == 1) {
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < psz; ++i)
        r[i] = -d_qm1 * o.vel_r[i] * gr[i] - d_qm1 * o.vel_t[i] * gt[i] - d_qm1 * o.vel_p[i] * gq[i];
    } else {
      const double Diss = d_qm1 * d_qm1 / o.cfg.Ra;
#pragma omp parallel for schedule(static)
      for (int n = 0; n < o.N; ++n) {
        const double xi0 = o.oc.rho1[n], T0 = o.oc.temp0[n], dT0 = o.oc.temp1[n], rho = o.oc.rho0[n];
        const double rrr = o.oc.R(n + 1, 1), eta = o.oc.eta0[n];
        for (size_t k = 0; k < (size_t)Th * Ph; ++k) {
          size_t i = k + (size_t)Th * Ph * n;
          double vr = o.vel_r[i], dur = o.vel_dur[i], qv1 = o.vel_qv1[i], qv2 = o.vel_qv2[i];
          double x = 2.0 * (dur * dur);
          double y = (xi0 + 1.0 / rrr) * vr + dur + qv1;
          x = x + 2.0 * (y * y);
          y = xi0 * vr;
          x = x - 2.0 * (y * y) / 3.0;
          y = qv1 + vr / rrr;
          x = x + 2.0 * (y * y);
          y = 2.0 * o.vel_dutr[i] - o.vel_cp[i];
          x = x + y * y;
          y = 2.0 * o.vel_dupr[i] + o.vel_ct[i];
          x = x + y * y;
          y = 2.0 * qv2 + o.vel_cr[i];
          x = x + y * y;
          double jr = o.mag_cr[i], jt = o.mag_ct[i], jp = o.mag_cp[i];
          x = x + eta * ((jr * jr + jp * jp + jt * jt) / (rho * o.cfg.E));
          double v = -(d_qm1 * vr * gr[i]) + (dT0 / T0) * gr[i];
          v = v - d_qm1 * o.vel_t[i] * gt[i];
          v = v - d_qm1 * o.vel_p[i] * gq[i];
          r[i] = v + (Diss / T0) * x;
        }
      }
    }
    Spec ss;
    tra_phys2spec(o, r, ss);
    Coll& NC = which == 0 ? o.codNC : o.compNC;
    spec2coll(o, ss, NC);
    double src = which == 0 ? o.cfg.source : o.cfg.source_comp;
    for (int n = 0; n < o.N; ++n) NC.re[n] = NC.re[n] + src;
  }
  // ---- non_magnetic (nonlinear.F90:363-473), insulating inner core
  {
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < psz; ++i) {
      r[i] = o.vel_t[i] * o.mag_p[i] - o.vel_p[i] * o.mag_t[i];
      th[i] = o.vel_p[i] * o.mag_r[i] - o.vel_r[i] * o.mag_p[i];
      ph[i] = o.vel_r[i] * o.mag_t[i] - o.vel_t[i] * o.mag_r[i];
    }
    Spec sq, ss, st;
    tra_rtp2qst(o, r, th, ph, sq, ss, st);
    Coll cq, cs, ct;
    spec2coll(o, sq, cq); spec2coll(o, ss, cs); spec2coll(o, st, ct);
    qstllcurlr(o, ct, o.bNPol);
    qstllcurlcurlr(o, cq, cs, o.bNTor);
    for (int n = 0; n < o.N; ++n) { o.bNTor.re[n] = 0; o.bNTor.im[n] = 0; o.bNPol.re[n] = 0; o.bNPol.im[n] = 0; }
  }
  // the inner core (nonlinear.F90:451-472): N = -rot_omega d/dphi of its field
  if (o.Nic > 1) {
    const int Ni = o.Nic;
    for (int part = 0; part < 2; ++part) {
      const Coll& a = part == 0 ? o.icTor : o.icPol;
      Coll& Nn = part == 0 ? o.icNTor : o.icNPol;
      for (int nh = 0; nh < o.H; ++nh) {
        const double m_ = (double)o.hm[nh];
        for (int n = 0; n < Ni; ++n) {
          const size_t i = (size_t)n + (size_t)Ni * nh;
          const double dre = -(a.im[i] * m_), dim = a.re[i] * m_;  // var_coll_dph
          Nn.re[i] = -o.rot_omega * dre;
          Nn.im[i] = -o.rot_omega * dim;
        }
      }
      for (int n = 0; n < Ni; ++n) { Nn.re[n] = 0.0; Nn.im[n] = 0.0; }
    }
  }
}

// non_rotation (nonlinear.F90:479-538): the viscous and magnetic torques on the inner core,
// surface integrals over r = r_i (tra_surfintegral, transform.fftw3.F90:1039-1062)
void non_rotation(Oracle& o) {
  const int Th = o.Th, Ph = o.Ph;
  const double vfac = o.oc.R(1, 3) * o.cfg.Pm, mfac = o.oc.R(1, 3) * 2 * o.cfg.Pm / o.cfg.E;
  auto surf = [&](auto f) {
    std::vector<double> Y(Th, 0.0);
    for (int m = 0; m < Ph; ++m)
      for (int j = 0; j < Th; ++j) Y[j] = Y[j] + f(j, (size_t)j + (size_t)Th * m);
    double S = 0.0;
    for (int j = 0; j < Th; ++j) S = S + Y[j] * o.gwP0[j];
    return S * 4.0 * d_PI / (double)Ph;
  };
  if (o.cfg.vel_bc > 2) {
    o.rot_velTorq = 0.0;
  } else {
    const double S = -2.0 / o.oc.R(1, 1);
    o.rot_velTorq = surf([&](int j, size_t i) { return (S * o.vel_p[i] - o.vel_ct[i]) * o.sn[j]; }) * vfac;
  }
  if (o.Nic == 1) o.rot_magTorq = 0.0;
  else o.rot_magTorq = surf([&](int j, size_t i) { return o.mag_r[i] * o.mag_p[i] * o.sn[j]; }) * mfac;
}
// rot_predictor / rot_corrector (rotation.F90:40-87)
void rot_predictor(Oracle& o) {
  if (o.cfg.rot_force_0) { o.rot_omega = 0.0; return; }
  o.rot_omega = o.rot_omega + (o.tim_dt / o.rot_inertia) * (o.rot_velTorq + o.rot_magTorq);
  o.sv_velTorq = o.rot_velTorq;
  o.sv_magTorq = o.rot_magTorq;
}
void rot_corrector(Oracle& o) {
  if (o.cfg.rot_force_0) return;
  o.rot_omega = o.rot_omega + (o.tim_dt * o.cfg.implicit / o.rot_inertia) *
                                  ((o.rot_velTorq + o.rot_magTorq) - (o.sv_velTorq + o.sv_magTorq));
  o.sv_velTorq = o.rot_velTorq;
  o.sv_magTorq = o.rot_magTorq;
}

// ---- predictor / corrector (velocity.F90:369-465, codensity.F90:224-259,
//      magnetic.F90:370-461) --------------------------------------------------------------
void vel_gre_adjust(const Oracle& o, Coll& Pol) {
  int N = o.N;
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh];
    if (l == 0) continue;
    const double* iG = &o.invG[(size_t)4 * l];
    const double* G1 = &o.Gre[(size_t)N * 2 * l];
    const double* G2 = G1 + N;
    for (int part = 0; part < 2; ++part) {
      double* x = part == 0 ? &Pol.re[(size_t)N * nh] : &Pol.im[(size_t)N * nh];
      double BCi = x[0], BCo = x[N - 1];
      double a = iG[0] * BCi + iG[2] * BCo;
      double b = iG[1] * BCi + iG[3] * BCo;
      for (int n = 0; n < N; ++n) x[n] = x[n] - a * G1[n] - b * G2[n];
    }
  }
}
void vel_setbc_Tor(const Oracle& o, Coll& a) {
  int N = o.N;
  const double rot_omega = o.rot_omega;
  for (int nh = 0; nh < o.H; ++nh) {
    a.re[(size_t)N * nh] = 0; a.re[(size_t)N * nh + N - 1] = 0;
    a.im[(size_t)N * nh] = 0; a.im[(size_t)N * nh + N - 1] = 0;
    if (o.cfg.vel_bc > 2) continue;
    if (o.hl[nh] != 1 || o.hm[nh] != 0) continue;
    a.re[(size_t)N * nh] = rot_omega * o.oc.R(1, nh);  // mes_oc%r(1,nh): nh is 1 here
    if (o.tim_it != 0) a.re[(size_t)N * nh] = a.re[(size_t)N * nh] - o.vTor.re[(size_t)N * nh];
  }
}
void scal_setbc(const Oracle& o, Coll& a, int bc, double qi, double qo) {
  int N = o.N;
  for (int nh = 0; nh < o.H; ++nh) {
    a.re[(size_t)N * nh] = 0; a.re[(size_t)N * nh + N - 1] = 0;
    a.im[(size_t)N * nh] = 0; a.im[(size_t)N * nh + N - 1] = 0;
  }
  if (bc == 1 || bc == 2) a.re[0] = 1.0;
  else if (bc == 3 || bc == 4) a.re[0] = qi;
  if (bc == 2 || bc == 4) a.re[N - 1] = qo;
  else a.re[N - 1] = 0.0;
}

void predictor(Oracle& o) {
  Coll T, Pq;
  if (o.cfg.rot_tstep) rot_predictor(o);  // main.F90:136, before vel_predictor's boundary value
  // vel_predictor
  o.sv_vNTor = o.vNTor;
  tim_multY(o, false, o.YTor, o.vTor, o.vNTor, T);
  vel_setbc_Tor(o, T);
  tim_invX(o, false, o.XTor, T);
  o.vTor = T;
  o.sv_vNPol = o.vNPol;
  Pq = o.vNPol;
  tim_zerobc(o, Pq);
  tim_invX(o, false, o.XGre, Pq);
  tim_multY(o, false, o.YPol, o.vPol, Pq, Pq);
  tim_zerobc(o, Pq);
  tim_invX(o, false, o.XPol, Pq);
  vel_gre_adjust(o, Pq);
  o.vPol = Pq;
  // cod_predictor
  o.sv_codNC = o.codNC;
  tim_multY(o, true, o.YC, o.codC, o.codNC, T);
  scal_setbc(o, T, o.cfg.cod_bc, o.cfg.qi, o.cfg.qo);
  tim_invX(o, true, o.XC, T);
  o.codC = T;
  if (o.cfg.comp_tstep) {
    o.sv_compNC = o.compNC;
    tim_multY(o, true, o.YComp, o.compC, o.compNC, T);
    scal_setbc(o, T, o.cfg.comp_bc, o.cfg.qi_comp, o.cfg.qo_comp);
    tim_invX(o, true, o.XComp, T);
    o.compC = T;
  }
  if (o.Nic > 1) {  // mag_predictor with the conducting inner core (magnetic.F90:370-408)
    Coll icT;
    for (int part = 0; part < 2; ++part) {
      const bool tor = part == 0;
      Coll& X = tor ? o.bTor : o.bPol;
      Coll& Nn = tor ? o.bNTor : o.bNPol;
      Coll& icX = tor ? o.icTor : o.icPol;
      Coll& icN = tor ? o.icNTor : o.icNPol;
      (tor ? o.sv_bNTor : o.sv_bNPol) = Nn;
      tim_multY(o, false, tor ? o.mYTor : o.mYPol, X, Nn, T);
      (tor ? o.sv_icNTor : o.sv_icNPol) = icN;
      tim_multY_n(o, o.Nic, false, tor ? o.icYTor : o.icYPol, icX, icN, icT);
      tim_zerobc_n(o, o.Nic, icT);
      tim_zerobc(o, T);  // mag_setbc_Tor / mag_setbc_Pol with zero boundary data
      tim_icinvX(o, tor ? o.mXTor : o.mXPol, T, icT);
      X = T;
      icX = icT;
    }
    return;
  }
  // mag_predictor (Ni = 1; zero toroidal/poloidal boundary data)
  o.sv_bNTor = o.bNTor;
  tim_multY(o, false, o.mYTor, o.bTor, o.bNTor, T);
  for (int nh = 0; nh < o.H; ++nh) {   // mag_setbc_Tor with zero BC arrays
    T.re[(size_t)o.N * nh + o.N - 1] = 0; T.im[(size_t)o.N * nh + o.N - 1] = 0;
    T.re[(size_t)o.N * nh] = 0; T.im[(size_t)o.N * nh] = 0;
  }
  tim_invX(o, false, o.mXTor, T);
  o.bTor = T;
  for (int nh = 0; nh < o.H; ++nh) {   // icTor(1,:) = oc solution at r_i
    if (o.hl[nh] == 0) continue;
    o.bicTor.re[(size_t)o.N * nh] = T.re[(size_t)o.N * nh]; o.bicTor.im[(size_t)o.N * nh] = T.im[(size_t)o.N * nh];
  }
  o.sv_bNPol = o.bNPol;
  tim_multY(o, false, o.mYPol, o.bPol, o.bNPol, T);
  for (int nh = 0; nh < o.H; ++nh) {   // mag_setbc_Pol with zero BC arrays
    T.re[(size_t)o.N * nh] = 0; T.im[(size_t)o.N * nh] = 0;
    T.re[(size_t)o.N * nh + o.N - 1] = 0; T.im[(size_t)o.N * nh + o.N - 1] = 0;
  }
  tim_invX(o, false, o.mXPol, T);
  o.bPol = T;
  for (int nh = 0; nh < o.H; ++nh) {
    if (o.hl[nh] == 0) continue;
    o.bicPol.re[(size_t)o.N * nh] = T.re[(size_t)o.N * nh]; o.bicPol.im[(size_t)o.N * nh] = T.im[(size_t)o.N * nh];
  }
}

void corrector(Oracle& o) {
  Coll T, Pq, ic;
  if (o.cfg.rot_tstep) rot_corrector(o);  // main.F90:148
  // vel_corrector
  tim_nlincorr(o, o.vNTor, o.sv_vNTor, T);
  o.sv_vNTor = o.vNTor;
  vel_setbc_Tor(o, T);
  tim_invX(o, false, o.XTor, T);
  tim_addcorr(o, T, o.vTor, o.N, o.N);
  tim_nlincorr(o, o.vNPol, o.sv_vNPol, Pq);
  o.sv_vNPol = o.vNPol;
  tim_zerobc(o, Pq);
  tim_invX(o, false, o.XGre, Pq);
  tim_zerobc(o, Pq);
  tim_invX(o, false, o.XPol, Pq);
  vel_gre_adjust(o, Pq);
  tim_addcorr(o, Pq, o.vPol, o.N, o.N);
  // cod_corrector
  tim_nlincorr(o, o.codNC, o.sv_codNC, T);
  o.sv_codNC = o.codNC;
  tim_zerobc(o, T);
  tim_invX(o, true, o.XC, T);
  tim_addcorr(o, T, o.codC, o.N, o.N);
  if (o.cfg.comp_tstep) {
    tim_nlincorr(o, o.compNC, o.sv_compNC, T);
    o.sv_compNC = o.compNC;
    tim_zerobc(o, T);
    tim_invX(o, true, o.XComp, T);
    tim_addcorr(o, T, o.compC, o.N, o.N);
  }
  if (o.Nic > 1) {  // mag_corrector with the conducting inner core (magnetic.F90:414-461)
    for (int part = 0; part < 2; ++part) {
      const bool tor = part == 0;
      const Coll& Nn = tor ? o.bNTor : o.bNPol;
      const Coll& icN = tor ? o.icNTor : o.icNPol;
      Coll& sv = tor ? o.sv_bNTor : o.sv_bNPol;
      Coll& icsv = tor ? o.sv_icNTor : o.sv_icNPol;
      tim_nlincorr(o, Nn, sv, T);
      sv = Nn;
      tim_nlincorr(o, icN, icsv, ic);
      icsv = icN;
      tim_zerobc_n(o, o.Nic, ic);
      tim_zerobc(o, T);
      tim_icinvX(o, tor ? o.mXTor : o.mXPol, T, ic);
      tim_addcorr(o, T, tor ? o.bTor : o.bPol, o.N, o.N);
      tim_addcorr(o, ic, tor ? o.icTor : o.icPol, o.Nic, o.Nic);
    }
    return;
  }
  // mag_corrector; with Ni = 1 the inner-core correction is row 1 of the outer-core one
  for (int part = 0; part < 2; ++part) {
    const Coll& Nn = part == 0 ? o.bNTor : o.bNPol;
    Coll& sv = part == 0 ? o.sv_bNTor : o.sv_bNPol;
    tim_nlincorr(o, Nn, sv, T);
    sv = Nn;
    tim_zerobc(o, T);  // mag_setbc_Tor (zero BC data) / tim_zerobc(Pol_p_m)
    tim_invX(o, false, part == 0 ? o.mXTor : o.mXPol, T);
    ic.init(o.N, o.H);
    for (int nh = 0; nh < o.H; ++nh) {
      if (o.hl[nh] == 0) continue;
      ic.re[(size_t)o.N * nh] = T.re[(size_t)o.N * nh]; ic.im[(size_t)o.N * nh] = T.im[(size_t)o.N * nh];
    }
    tim_addcorr(o, T, part == 0 ? o.bTor : o.bPol, o.N, o.N);
    tim_addcorr(o, ic, part == 0 ? o.bicTor : o.bicPol, 1, o.N);
  }
}

// non_maxtstep (nonlinear.F90:546-615): the CFL limit from u and B on the grid
void non_maxtstep(Oracle& o) {
  const int N = o.N, Th = o.Th, Ph = o.Ph;
  const double E = o.cfg.E, Pm = o.cfg.Pm;
  o.tim_cfl_dt = 1e99;
  for (int n = 1; n <= N; ++n) {
    double dr;
    if (n == 1) dr = o.oc.R(2, 1) - o.oc.R(1, 1);
    else if (n == N) dr = o.oc.R(N, 1) - o.oc.R(N - 1, 1);
    else dr = std::min(o.oc.R(n, 1) - o.oc.R(n - 1, 1), o.oc.R(n + 1, 1) - o.oc.R(n, 1));
    double d = (E + E / Pm) / (2.0 * dr);
    d = d * d;
    double mx = -1e300;
    const size_t base = (size_t)Th * Ph * (n - 1);
    for (size_t k = 0; k < (size_t)Th * Ph; ++k) {
      double p = o.mag_r[base + k] * o.mag_r[base + k];
      double v = p / std::sqrt(p * (E / Pm) + d) + std::fabs(o.vel_r[base + k]);
      mx = std::max(mx, v);
    }
    if (mx != 0.0) o.tim_cfl_dt = std::min(o.tim_cfl_dt, dr / mx);
    dr = o.oc.R(n, 1) / std::sqrt((double)(o.L * (o.L - 1)));
    d = E / (2.0 * dr);
    d = d * d;
    mx = -1e300;
    for (size_t k = 0; k < (size_t)Th * Ph; ++k) {
      double p = o.mag_t[base + k] * o.mag_t[base + k] + o.mag_p[base + k] * o.mag_p[base + k];
      double vt = o.vel_t[base + k], vp = o.vel_p[base + k];
      double v = p / std::sqrt(p * E / Pm + d) + std::sqrt(vt * vt + vp * vp);
      mx = std::max(mx, v);
    }
    if (mx != 0.0) o.tim_cfl_dt = std::min(o.tim_cfl_dt, dr / mx);
  }
  o.tim_cfl_dt = std::min(o.tim_cfl_dt, E / Pm);
  o.tim_cfl_dt = std::min(o.tim_cfl_dt, std::sqrt(E));
}
// tim_new_tstep (timestep.F90:837-870); O: anything with the tim_* members and cfg
template <class O>
void tim_new_tstep(O& o) {
  double dt = o.tim_dt;
  if (o.cfg.time_step_control == 1) {
    if (o.tim_corr_dt > o.cfg.corr_upper) dt = 0.5 * dt;
    if (o.tim_corr_dt < o.cfg.corr_lower) dt = 1.273974 * dt;
    if (o.tim_step == 0) dt = std::min(dt / 1e3, 1e-8);
  } else {
    if (o.tim_corr_dt > 0.0) dt = std::min(o.tim_corr_dt, dt * 2.0 / o.cfg.courant);
    if (o.tim_cfl_dt > 0.0) dt = std::min(o.tim_cfl_dt, dt);
    if (o.tim_step == 0) dt = std::min(dt / 1e3, 1e-10);
    dt = dt * o.cfg.courant;
  }
  o.tim_new_dt = (dt < o.tim_dt * 0.97 || dt > o.tim_dt * 1.03);
  if (o.tim_new_dt) o.tim_dt = dt;
}

// tim_check_cgce (timestep.F90:744-830); returns 1 when the loop gave up.
template <class O>
int check_cgce(O& o) {
  int fail = 0;
  const int i_maxtstep = 1500000;
  if (o.cfg.time_step_control == 1) {
    if (o.tim_it == 1) { o.tim_corr_dt = o.tim_dterr; o.lasterr = 1e99; }
    if (o.tim_dt < 1e-12 && o.tim_step > 30) { o.tim_step = i_maxtstep - 1; o.tim_it = 0; fail = 1; }
    else if (o.tim_it > 10) { o.tim_step = i_maxtstep - 1; o.tim_it = 0; fail = 1; }
    else if (o.tim_dterr > o.lasterr) { if (o.tim_dterr > 1.0) fail = 1; o.tim_it = 0; }
    else if (o.tim_dterr > 1.0) { o.lasterr = o.tim_dterr; o.tim_it = o.tim_it + 1; }
    else o.tim_it = 0;
    o.tim_dterr = 0.0;
  } else {
    if (o.tim_it == 1) { o.tim_corr_dt = o.tim_dt * std::sqrt(o.cfg.dterr / o.tim_dterr); o.lasterr = 1e99; }
    if (o.tim_dt < 1e-12 && o.tim_step > 30) { o.tim_it = 0; fail = 1; }
    else if (o.tim_it == o.tim_pcn) o.tim_it = 0;
    else if (o.tim_it > 10) { o.tim_it = 0; fail = 1; }
    else if (o.tim_dterr > o.lasterr) {
      if (o.tim_dterr > 2.0 * o.cfg.dterr) fail = 1;
      if (o.tim_dterr < 2.0 * o.cfg.dterr) o.tim_corr_dt = o.tim_dt / (1e1 * o.cfg.courant);
      o.tim_it = 0;
    } else if (o.tim_dterr > o.cfg.dterr) { o.lasterr = o.tim_dterr; o.tim_it = o.tim_it + 1; }
    else o.tim_it = 0;
    o.tim_dterr = 0.0;
  }
  return fail;
}

// ========================================================================================
// Energies (io.F90:1739-2024, variables.F90:903-957, 1118-1170)
// ========================================================================================
// var_coll_norm / _norm_comp / _norm_magdiss differ only in the radial weights
void coll_norm_w(const Oracle& o, const Coll& a, const std::vector<double>& wts, double& Eodd, double& Eeven,
                 double& Em0le, double& Em0);
void coll_norm(const Oracle& o, const Coll& a, double& Eodd, double& Eeven, double& Em0le, double& Em0) {
  coll_norm_w(o, a, o.oc.intr2dr, Eodd, Eeven, Em0le, Em0);
}
void coll_norm_n(const Oracle& o, int N, const Coll& a, const std::vector<double>& wts, double& Eodd,
                 double& Eeven, double& Em0le, double& Em0);
void coll_norm_w(const Oracle& o, const Coll& a, const std::vector<double>& wts, double& Eodd, double& Eeven,
                 double& Em0le, double& Em0) {
  coll_norm_n(o, o.N, a, wts, Eodd, Eeven, Em0le, Em0);
}
void coll_norm_n(const Oracle& o, int N, const Coll& a, const std::vector<double>& wts, double& Eodd,
                 double& Eeven, double& Em0le, double& Em0) {
  std::vector<double> Fod(N, 0), Fev(N, 0), Fm0le(N, 0), Fm0(N, 0), f(N);
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh], m_ = o.hm[nh];
    double w = 4.0 * d_PI / (double)(2 * l + 1);
    if (m_ != 0) w = 4.0 * w;
    for (int n = 0; n < N; ++n) {
      size_t i = n + (size_t)N * nh;
      f[n] = w * (a.re[i] * a.re[i] + a.im[i] * a.im[i]);
    }
    if (m_ == 0) for (int n = 0; n < N; ++n) Fm0[n] = Fm0[n] + f[n];
    if (m_ == 0 && l % 2 == 0) for (int n = 0; n < N; ++n) Fm0le[n] = Fm0le[n] + f[n];
    if (((l - m_) % 2 + 2) % 2 == 1) for (int n = 0; n < N; ++n) Fod[n] = Fod[n] + f[n];
    else for (int n = 0; n < N; ++n) Fev[n] = Fev[n] + f[n];
  }
  auto dot = [&](const std::vector<double>& v) { double s = 0; for (int n = 0; n < N; ++n) s = s + v[n] * wts[n]; return s; };
  Eodd = dot(Fod); Eeven = dot(Fev); Em0le = dot(Fm0le); Em0 = dot(Fm0);
}
// var_coll_norm_veldiss (variables.F90:1034-1061)
double coll_norm_veldiss(const Oracle& o, const Coll& a) {
  int N = o.N;
  std::vector<double> F(N, 0.0);
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh], m_ = o.hm[nh];
    double w = 4.0 * d_PI / (double)(2 * l + 1);
    if (m_ != 0) w = 4.0 * w;
    for (int n = 0; n < N; ++n) {
      size_t i = n + (size_t)N * nh;
      F[n] = F[n] + w * (a.re[i] * a.re[i] + a.im[i] * a.im[i]);
    }
  }
  double s = 0;
  for (int n = 0; n < N; ++n) s = s + F[n] * o.oc.intr2dr_veldiss[n];
  return s;
}
double coll_norm_surf_in(const Oracle& o, const Coll& a, bool outer) {
  int N = o.N;
  double F = 0;
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh], m_ = o.hm[nh];
    double w = 4.0 * d_PI / (double)(2 * l + 1);
    if (m_ != 0) w = 4.0 * w;
    size_t i = (outer ? N - 1 : 0) + (size_t)N * nh;
    F = F + w * (a.re[i] * a.re[i] + a.im[i] * a.im[i]);
  }
  if (!o.cfg.boussinesq) return F * o.oc.rho0[outer ? N - 1 : 0] * o.oc.R(outer ? N : 1, 1);
  return F * o.oc.R(outer ? N : 1, 1);
}

void energies(Oracle& o, double* out) {
  for (int i = 0; i < LSD_NENERGY; ++i) out[i] = 0.0;
  out[LSD_E_TIME] = o.tim_t;
  // io_write2files prefactors (io.F90:234-247)
  const bool bq = o.cfg.boussinesq != 0;
  double KE = 0.5, VD = o.cfg.Pm, ME = 0.5 * o.cfg.Pm / o.cfg.E, OD = 1.0 * o.cfg.Pm / o.cfg.E;
  if (bq) { ME = o.cfg.Pm / o.cfg.E; OD = 2.0 * o.cfg.Pm / o.cfg.E; }
  const std::vector<double>& wv = bq ? o.oc.intr2dr : o.oc.intr2dr_comp;
  int N = o.N, KL = o.KL;
  // heat fluxes (io.F90:1773-1794)
  double flx = 0;
  for (int j = N - KL; j <= N; ++j) flx = flx - o.codC.re[j - 1] * o.oc.dr[1].at(KL + 1 + N - j, j);
  if (bq) out[LSD_E_TOPFLX] = 4.0 * d_PI * o.oc.R(N, 2) * flx;
  else out[LSD_E_TOPFLX] = 4.0 * d_PI * o.oc.R(N, 2) * o.oc.rho0[N - 1] * o.oc.temp0[N - 1] * flx;
  flx = 0;
  for (int j = 1; j <= 1 + KL; ++j) flx = flx - o.codC.re[j - 1] * o.oc.dr[1].at(KL + 2 - j, j);
  if (bq) out[LSD_E_BOTFLX] = 4.0 * d_PI * o.oc.R(1, 2) * flx;
  else out[LSD_E_BOTFLX] = 4.0 * d_PI * o.oc.R(1, 2) * o.oc.rho0[0] * o.oc.temp0[0] * flx;
  // velocity
  {
    Coll q, s, t;
    torpol2qst(o, o.vTor, o.vPol, q, s, t, true);
    double Eo, Ee, E1, E0, Ep, Epas, Esym, El1, Et, Etas;
    coll_norm_w(o, q, wv, Eo, Ee, E1, E0);
    double ESin = coll_norm_surf_in(o, q, false), ESout = coll_norm_surf_in(o, q, true);
    const double Ecomp = bq ? 0.0 : coll_norm_veldiss(o, q);
    Ep = Eo + Ee; Epas = E0; Esym = Ee; El1 = E1;
    coll_norm_w(o, s, wv, Eo, Ee, E1, E0);
    ESin = ESin + coll_norm_surf_in(o, s, false); ESout = ESout + coll_norm_surf_in(o, s, true);
    Ep = Ep + Eo + Ee; Epas = Epas + E0; Esym = Esym + Ee; El1 = El1 + E1;
    coll_norm_w(o, t, wv, Eo, Ee, E1, E0);
    ESin = ESin + coll_norm_surf_in(o, t, false); ESout = ESout + coll_norm_surf_in(o, t, true);
    Et = Eo + Ee; Etas = E0; Esym = Esym + Eo; El1 = El1 + E1;
    qstcurl(o, q, s, t, q, s, t);
    double EDis;
    coll_norm_w(o, q, wv, Eo, Ee, E1, E0); EDis = Eo + Ee;
    coll_norm_w(o, s, wv, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    coll_norm_w(o, t, wv, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    double ETm0 = KE * E0;
    out[LSD_E_KE] = KE * (Ep + Et);
    out[LSD_E_KE_TOR] = KE * Et;
    out[LSD_E_KE_SYM] = KE * Esym;
    out[LSD_E_KE_L1] = KE * El1;
    out[LSD_E_KE_TM0] = ETm0;
    out[LSD_E_KE_DIS] = VD * EDis + VD * 2.0 * (ESin - ESout) + Ecomp;
    out[LSD_E_KE_AX] = KE * Epas + KE * Etas;
  }
  // magnetic
  {
    Coll q, s, t;
    torpol2qst(o, o.bTor, o.bPol, q, s, t, false);
    double Eo, Ee, E1, E0, Ep, Epas, Esym, El1, Et, Etas, ETm0;
    coll_norm(o, q, Eo, Ee, E1, E0);
    Ep = Eo + Ee; Epas = E0; Esym = Ee; El1 = E1;
    coll_norm(o, s, Eo, Ee, E1, E0);
    Ep = Ep + Eo + Ee; Epas = Epas + E0; Esym = Esym + Ee; El1 = El1 + E1;
    coll_norm(o, t, Eo, Ee, E1, E0);
    Et = Eo + Ee; Etas = E0; ETm0 = E0; Esym = Esym + Eo; El1 = El1 + E1;
    qstcurl(o, q, s, t, q, s, t);
    double EDis;  // var_coll_norm_magdiss
    coll_norm_w(o, q, o.oc.intr2dr_magdiss, Eo, Ee, E1, E0); EDis = Eo + Ee;
    coll_norm_w(o, s, o.oc.intr2dr_magdiss, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    coll_norm_w(o, t, o.oc.intr2dr_magdiss, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    out[LSD_E_ME] = ME * (Ep + Et);
    out[LSD_E_ME_TOR] = ME * Et;
    out[LSD_E_ME_SYM] = ME * Esym;
    out[LSD_E_ME_L1] = ME * El1;
    out[LSD_E_ME_TM0] = ME * ETm0;
    out[LSD_E_ME_DIS] = OD * EDis;
    out[LSD_E_DIP] = o.bPol.re[(size_t)N * 1 + N - 1] / o.oc.R(N, 1);
    out[LSD_E_QUAD] = 2 * o.bPol.re[(size_t)N * 2 + N - 1] / o.oc.R(N, 1);
    out[LSD_E_ME_AX] = ME * Etas + ME * Epas;
  }
}

// ========================================================================================
// The other diagnostics of io_write2files (io.F90:1739-2738)
// ========================================================================================
// var_coll_normlm / _normlm_comp (variables.F90:1267-1364): per-l and per-m energies
void normlm(const Oracle& o, const Coll& a, const std::vector<double>& wts, std::vector<double>& El,
            std::vector<double>& Em) {
  const int N = o.N;
  El.assign(o.L, 0.0); Em.assign(o.M, 0.0);
  std::vector<double> f(N);
  for (int nh = 0; nh < o.H; ++nh) {
    int l = o.hl[nh], m = o.hm[nh] / o.Mp;
    double w = 4.0 * d_PI / (double)(2 * l + 1);
    if (m != 0) w = 4.0 * w;
    double e = 0.0;
    for (int n = 0; n < N; ++n) {
      size_t i = n + (size_t)N * nh;
      f[n] = w * (a.re[i] * a.re[i] + a.im[i] * a.im[i]);
      e = e + f[n] * wts[n];
    }
    El[l] = El[l] + e;
    Em[m] = Em[m] + e;
  }
}
// meshmult of dr(1) at row n (1-based) of column nh (Re part)
double dr1_row(const Oracle& o, const Coll& a, int nh, int n) {
  const int N = o.N, KL = o.KL;
  double acc = 0.0;
  for (int j = std::max(1, n - KL); j <= std::min(n + KL, N); ++j)
    acc = acc + o.oc.dr[1].at(KL + 1 + n - j, j) * a.re[(j - 1) + (size_t)N * nh];
  return acc;
}
// io_write_nussel (io.F90:2158-2243)
void nusselt(const Oracle& o, const Coll& C, double* out) {
  const int N = o.N;
  const double T_ri = C.re[0], T_ro = C.re[N - 1];
  const double dCdr_ri = dr1_row(o, C, 0, 1), dCdr_ro = dr1_row(o, C, 0, N);
  const double ri = o.cfg.rratio / (1 - o.cfg.rratio), ro = 1 / (1 - o.cfg.rratio);
  const double A = (ri * ro) / (ri - ro);
  double nu_top = 0, nu_bot = 0, nu_flux = 0, nu = 0;
  if (o.cfg.cod_bc == 1) {
    nu_bot = dCdr_ri / (A / (ri * ri));
    nu_top = dCdr_ro / (A / (ro * ro));
    nu = nu_top;
  } else if (o.cfg.cod_bc == 4) {
    const double DT_cond = 1 / ri - 1 / ro, DT = T_ri - T_ro;
    nu_flux = DT_cond / DT;
    nu = nu_flux;
  }
  const double v[8] = {nu, T_ro, T_ri, dCdr_ri, dCdr_ro, nu_top, nu_bot, nu_flux};
  for (int k = 0; k < 8; ++k) out[k] = v[k];
}

void diagnostics(Oracle& o, double* sc, double* spec, double* prof) {
  const bool bq = o.cfg.boussinesq != 0;
  const int N = o.N, L = o.L, M = o.M;
  const double KE = 0.5;
  double ME = 0.5 * o.cfg.Pm / o.cfg.E;
  if (bq) ME = o.cfg.Pm / o.cfg.E;
  for (int i = 0; i < LSD_NDIAG; ++i) sc[i] = 0.0;
  sc[LSD_D_TIME] = o.tim_t;
  double en[LSD_NENERGY];
  energies(o, en);
  const std::vector<double>& w2 = o.oc.intr2dr;
  const std::vector<double>& wv = bq ? o.oc.intr2dr : o.oc.intr2dr_comp;
  // ---- velocity: compressible q, s, t (io_write_vel_energy, io_rad_profile)
  Coll q, s, t, qm, sm, tm;
  torpol2qst(o, o.vTor, o.vPol, q, s, t, true);
  torpol2qst(o, o.vTor, o.vPol, qm, sm, tm, false);
  {
    double Eo, Ee, E1, E0, Ep, Epes, Epesas, Epas, Et, Etes, Etesas, Etas;
    coll_norm_w(o, q, wv, Eo, Ee, E1, E0); Ep = Eo + Ee; Epes = Ee; Epesas = E1; Epas = E0;
    coll_norm_w(o, s, wv, Eo, Ee, E1, E0); Ep = Ep + Eo + Ee; Epes = Epes + Ee; Epesas = Epesas + E1; Epas = Epas + E0;
    coll_norm_w(o, t, wv, Eo, Ee, E1, E0); Et = Eo + Ee; Etes = Eo; Etesas = E0 - E1; Etas = E0;
    std::vector<double> ETl, ETm, EQl, EQm, ESl, ESm;
    normlm(o, t, w2, ETl, ETm); normlm(o, q, w2, EQl, EQm); normlm(o, s, w2, ESl, ESm);
    double l_Eofl = 0.0;
    for (int i = 1; i < L; ++i) l_Eofl = l_Eofl + i * KE * (ETl[i] + EQl[i] + ESl[i]);
    int lpol = 0;
    double best = -1.0;
    for (int i = 0; i < L; ++i) if (EQl[i] + ESl[i] > best) { best = EQl[i] + ESl[i]; lpol = i + 1; }
    const double v[10] = {KE * Et, KE * Ep, KE * Etas, KE * Epas, KE * Etes, KE * Epes, KE * Etesas, KE * Epesas,
                          l_Eofl, (double)lpol};
    for (int k = 0; k < 10; ++k) sc[LSD_D_VPART + k] = v[k];
  }
  // ---- field: q, s, t of var_coll_TorPol2qst_mag (io_write_mag_energy)
  Coll bq_, bs_, bt_, bcq, bcs, bct;
  torpol2qst(o, o.bTor, o.bPol, bq_, bs_, bt_, false);
  torpol2qst(o, o.bTor, o.bPol, bcq, bcs, bct, true);  // io_rad_profile, io_write_cmb
  {
    double Eo, Ee, E1, E0, Ep, Epes, Epesas, Epas, Et, Etes, Etesas, Etas;
    coll_norm(o, bq_, Eo, Ee, E1, E0); Ep = Eo + Ee; Epes = Ee; Epesas = E1; Epas = E0;
    coll_norm(o, bs_, Eo, Ee, E1, E0); Ep = Ep + Eo + Ee; Epes = Epes + Ee; Epesas = Epesas + E1; Epas = Epas + E0;
    coll_norm(o, bt_, Eo, Ee, E1, E0); Et = Eo + Ee; Etes = Eo; Etesas = E0 - E1; Etas = E0;
    const double v[8] = {ME * Et, ME * Ep, ME * Etas, ME * Epas, ME * Etes, ME * Epes, ME * Etesas, ME * Epesas};
    for (int k = 0; k < 8; ++k) sc[LSD_D_MPART + k] = v[k];
  }
  // ---- the inner core's field (io_write_mag_energy on mag_icTor / icPol, io.F90:315):
  // its own mesh, the outer core's Dip / Quad; the call leaves io_MagEn / io_OhmDiss at
  // the inner core's values for io_write_dyn_outputs
  double icE = 0.0, icEDis = 0.0;
  if (o.Nic > 1) {
    const RDom& I = o.ic;
    const int Ni = o.Nic;
    const double OD = bq ? 2.0 * o.cfg.Pm / o.cfg.E : 1.0 * o.cfg.Pm / o.cfg.E;
    Coll q, s, t, cq, cs, ct;
    torpol2qst_d(o, I, o.icTor, o.icPol, q, s, t, false);
    double Eo, Ee, E1, E0, Ep, Epes, Epesas, Epas, Et, Etes, Etesas, Etas, Esym, El1, ETm0, EDis;
    coll_norm_n(o, Ni, q, I.intr2dr, Eo, Ee, E1, E0);
    Ep = Eo + Ee; Epes = Ee; Epesas = E1; Epas = E0; Esym = Ee; El1 = E1;
    coll_norm_n(o, Ni, s, I.intr2dr, Eo, Ee, E1, E0);
    Ep = Ep + Eo + Ee; Epes = Epes + Ee; Epesas = Epesas + E1; Epas = Epas + E0; Esym = Esym + Ee; El1 = El1 + E1;
    coll_norm_n(o, Ni, t, I.intr2dr, Eo, Ee, E1, E0);
    Et = Eo + Ee; Etes = Eo; Etesas = E0 - E1; Etas = E0; ETm0 = E0; Esym = Esym + Eo; El1 = El1 + E1;
    qstcurl_d(o, I, q, s, t, cq, cs, ct);
    coll_norm_n(o, Ni, cq, I.intr2dr_magdiss, Eo, Ee, E1, E0); EDis = Eo + Ee;
    coll_norm_n(o, Ni, cs, I.intr2dr_magdiss, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    coll_norm_n(o, Ni, ct, I.intr2dr_magdiss, Eo, Ee, E1, E0); EDis = EDis + Eo + Ee;
    icE = ME * (Ep + Et);
    icEDis = OD * EDis;
    const double v[9] = {icE, ME * Et, ME * Esym, ME * El1, ME * ETm0, icEDis, en[LSD_E_DIP], en[LSD_E_QUAD],
                         ME * Etas + ME * Epas};
    for (int k = 0; k < 9; ++k) sc[LSD_D_MIC + k] = v[k];
    const double w[8] = {ME * Et, ME * Ep, ME * Etas, ME * Epas, ME * Etes, ME * Epes, ME * Etesas, ME * Epesas};
    for (int k = 0; k < 8; ++k) sc[LSD_D_MICPART + k] = w[k];
  }
  sc[LSD_D_ROT + 0] = o.rot_omega; sc[LSD_D_ROT + 1] = o.rot_velTorq; sc[LSD_D_ROT + 2] = o.rot_magTorq;
  // ---- CMB (io_write_cmb): the norms of q, s on the outer shell only
  double fdip = 0.0, thdip = 0.0;
  {
    double EPol = 0, ESym = 0, El1 = 0, Epas = 0, El12 = 0;
    for (const Coll* a : {&bcq, &bcs}) {
      double Fod = 0, Fev = 0, Fl1 = 0, Fm0 = 0, Fl12 = 0;
      for (int nh = 0; nh < o.H; ++nh) {
        int l = o.hl[nh], m_ = o.hm[nh];
        double w = 4.0 * d_PI / (double)(2 * l + 1);
        if (m_ != 0) w = 4.0 * w;
        size_t i = (N - 1) + (size_t)N * nh;
        double f = w * (a->re[i] * a->re[i] + a->im[i] * a->im[i]);
        if (m_ == 0) Fm0 = Fm0 + f;
        if (l > 0 && l <= 12) Fl12 = Fl12 + f;
        if (l == 1) Fl1 = Fl1 + f;
        if (((l - m_) % 2 + 2) % 2 == 1) Fod = Fod + f; else Fev = Fev + f;
      }
      const double wN = w2[N - 1];
      EPol = EPol + Fod * wN + Fev * wN;
      ESym = ESym + Fev * wN;
      El1 = El1 + Fl1 * wN;
      Epas = Epas + Fm0 * wN;
      El12 = El12 + Fl12 * wN;
    }
    const double fac = o.oc.R(N, 2) / w2[N - 1];
    EPol = ME * EPol * fac; Epas = ME * Epas * fac; ESym = ME * ESym * fac; El1 = ME * El1 * fac; El12 = ME * El12 * fac;
    int nh10 = 0, nh11 = -1;
    for (int nh = 0; nh < o.H; ++nh) {
      if (o.hl[nh] == 1 && o.hm[nh] == 0) nh10 = nh;
      if (o.hl[nh] == 1 && o.hm[nh] == 1) nh11 = nh;
    }
    const double g10 = o.bPol.re[(N - 1) + (size_t)N * nh10];
    double th, ph;
    if (o.Mp == 1 && o.M > 1 && nh11 >= 0) {
      const double g11 = -2.0 * o.bPol.re[(N - 1) + (size_t)N * nh11];
      const double h11 = 2.0 * o.bPol.im[(N - 1) + (size_t)N * nh11];
      th = std::sqrt(g10 * g10 + g11 * g11 + h11 * h11);
      if (th != 0.0) th = std::acos(g10 / std::max(th, std::fabs(g10)));
      if (std::fabs(g11) < 1e-99) ph = h11 >= 0.0 ? 0.5 * d_PI : 1.5 * d_PI;
      else {
        ph = std::atan(h11 / g11);
        if (g11 < 0.0) ph = ph + d_PI;
        if (ph < 0.0) ph = ph + 2.0 * d_PI;
      }
    } else {
      th = g10 >= 0.0 ? 0.0 : d_PI;
      ph = 0.0;
    }
    fdip = std::sqrt(El1 / El12);
    thdip = th;
    const double v[7] = {EPol, ESym, El1, th, ph, Epas, El12};
    for (int k = 0; k < 7; ++k) sc[LSD_D_CMB + k] = v[k];
  }
  // ---- Nusselt numbers (codensity, composition)
  nusselt(o, o.codC, sc + LSD_D_NUSC);
  if (o.cfg.comp_tstep) nusselt(o, o.compC, sc + LSD_D_NUSX);
  // ---- io_write_dyn_outputs
  {
    const double ri = o.cfg.rratio / (1 - o.cfg.rratio), ro = 1 / (1 - o.cfg.rratio);
    const double vol = (4.0 / 3.0 * d_PI) * (ro * ro * ro - ri * ri * ri);
    const double Kin = en[LSD_E_KE], Visc = en[LSD_E_KE_DIS];
    const double Mag = o.Nic > 1 ? icE : en[LSD_E_ME], Ohm = o.Nic > 1 ? icEDis : en[LSD_E_ME_DIS];
    const double Rm = std::sqrt((2 * Kin) / vol), Re = Rm / o.cfg.Pm;
    const double El = (o.cfg.E * Mag) / (o.cfg.Pm * vol);
    const double Le = std::sqrt((2 * o.cfg.E * o.cfg.E * Mag) / (o.cfg.Pm * o.cfg.Pm * vol));
    const double v[13] = {Rm, Re, Re * o.cfg.Pr, Re * o.cfg.Sc, Re * o.cfg.E, Mag / Kin, El, Le, fdip,
                          Ohm / (Ohm + Visc), thdip, sc[LSD_D_NUSC], o.cfg.comp_tstep ? sc[LSD_D_NUSX] : 0.0};
    for (int k = 0; k < 13; ++k) sc[LSD_D_DYN + k] = v[k];
  }
  sc[LSD_D_DT + 0] = o.tim_dt; sc[LSD_D_DT + 1] = o.tim_corr_dt; sc[LSD_D_DT + 2] = o.tim_cfl_dt;
  // ---- spectra
  if (spec) {
    double* p = spec;
    auto vec_spec = [&](const Coll& a, const Coll& b, const Coll& c, const std::vector<double>& wt, double Efac) {
      std::vector<double> ETl, ETm, EQl, EQm, ESl, ESm;
      normlm(o, c, wt, ETl, ETm); normlm(o, a, wt, EQl, EQm); normlm(o, b, wt, ESl, ESm);
      for (int l = 0; l < L; ++l) {
        *p++ = Efac * (ETl[l] + EQl[l] + ESl[l]); *p++ = Efac * (EQl[l] + ESl[l]); *p++ = Efac * ETl[l];
      }
      for (int m = 0; m < M; ++m) {
        *p++ = Efac * (ETm[m] + EQm[m] + ESm[m]); *p++ = Efac * (EQm[m] + ESm[m]); *p++ = Efac * ETm[m];
      }
    };
    if (bq) vec_spec(qm, sm, tm, w2, KE);
    else vec_spec(q, s, t, o.oc.intr2dr_comp, KE);  // io_save_spectrum_anelastic
    vec_spec(bq_, bs_, bt_, w2, ME);
    for (const Coll* a : {&o.codC, &o.compC}) {
      std::vector<double> El, Em;
      normlm(o, *a, w2, El, Em);
      for (int l = 0; l < L; ++l) *p++ = El[l];
      for (int m = 0; m < M; ++m) *p++ = Em[m];
    }
  }
  // ---- profiles
  if (prof) {
    for (int n = 0; n < N; ++n) prof[n] = o.oc.R(n + 1, 1);
    auto rad = [&](const Coll& a, const Coll& b, const Coll& c, double Efac, double* out) {
      std::vector<double> Ep(N, 0.0), Et(N, 0.0);
      for (int nh = 0; nh < o.H; ++nh) {
        int l = o.hl[nh], m_ = o.hm[nh];
        double w = 4.0 * d_PI / (double)(2 * l + 1);
        if (m_ != 0) w = 4.0 * w;
        for (int n = 0; n < N; ++n) {
          size_t i = n + (size_t)N * nh;
          double eq = w * (a.re[i] * a.re[i] + a.im[i] * a.im[i]);
          double es = w * (b.re[i] * b.re[i] + b.im[i] * b.im[i]);
          double et = w * (c.re[i] * c.re[i] + c.im[i] * c.im[i]);
          Ep[n] = Ep[n] + eq + es;
          Et[n] = Et[n] + et;
        }
      }
      for (int n = 0; n < N; ++n) {
        out[N + n] = Efac * Ep[n];
        out[2 * N + n] = Efac * Et[n];
        out[n] = out[2 * N + n] + out[N + n];
      }
    };
    rad(q, s, t, KE, prof + N);
    rad(bcq, bcs, bct, ME, prof + 4 * N);
    for (int k = 0; k < 2; ++k) {
      const Coll& C = k == 0 ? o.codC : o.compC;
      for (int n = 0; n < N; ++n) {
        prof[(7 + 2 * k) * N + n] = C.re[n];
        prof[(8 + 2 * k) * N + n] = dr1_row(o, C, 0, n + 1);
      }
    }
  }
}

Coll* field_ptr(Oracle& o, int f) {
  switch (f) {
    case LSD_VEL_TOR: return &o.vTor;
    case LSD_VEL_POL: return &o.vPol;
    case LSD_COD_C: return &o.codC;
    case LSD_MAG_TOR: return &o.bTor;
    case LSD_MAG_POL: return &o.bPol;
    case LSD_COMP_C: return &o.compC;
    case LSD_MAG_IC_TOR: return o.Nic > 1 ? &o.icTor : nullptr;
    case LSD_MAG_IC_POL: return o.Nic > 1 ? &o.icPol : nullptr;
  }
  return nullptr;
}
Coll* nl_ptr(Oracle& o, int f) {
  switch (f) {
    case LSD_N_VEL_TOR: return &o.vNTor;
    case LSD_N_VEL_POL: return &o.vNPol;
    case LSD_N_COD: return &o.codNC;
    case LSD_N_MAG_TOR: return &o.bNTor;
    case LSD_N_MAG_POL: return &o.bNPol;
    case LSD_N_COMP: return &o.compNC;
  }
  return nullptr;
}

}  // namespace

// ========================================================================================
// C entry points (mirroring include/lsd_b200.h with an orc_ prefix)
// ========================================================================================
extern "C" {

int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

Oracle* orc_create(const lsd_config* cfg, int* status) {
  Oracle* o = new Oracle();
  o->cfg = *cfg;
  o->L = cfg->L; o->M = cfg->M; o->Mp = cfg->Mp; o->N = cfg->N; o->KL = cfg->KL; o->Nic = cfg->Nic;
  *status = 0;
  const bool cic_ok = o->Nic == 1 || (o->Nic >= 2 * o->KL + 1 && o->Nic <= o->N && cfg->boussinesq &&
                                       cfg->vel_bc <= 2);
  if (o->L <= (o->M - 1) * o->Mp || (o->M > 1 && o->M % 2 == 1) || o->N < 2 * o->KL + 1 || !cic_ok ||
      (cfg->rot_tstep && !cfg->boussinesq) || cfg->timestep == 0) {
    *status = LSD_EARG;
    delete o;
    return nullptr;
  }
  o->Ma = o->M * 3 / 2;
  o->H = o->L * o->M - o->Mp * (o->M - 1) * o->M / 2;
  o->Th = o->L * 3 / 2;
  o->Th2 = (o->Th + 1) / 2;
  o->Ph = o->Ma * 2;
  o->Hc = (o->M + 1) / 2;
  o->Hr = o->H / o->Hc;
  o->tim_dt = cfg->timestep < 0 ? -cfg->timestep : cfg->timestep;
  setup_layout(*o);
  if (setup_legendre(*o) || setup_mesh(*o)) { *status = LSD_ESINGULAR; delete o; return nullptr; }
  o->fft.init(o->Ph);
  for (Coll* c : {&o->vTor, &o->vPol, &o->codC, &o->compC, &o->bTor, &o->bPol, &o->bicTor, &o->bicPol,
                  &o->vNTor, &o->vNPol, &o->codNC, &o->compNC, &o->bNTor, &o->bNPol,
                  &o->sv_vNTor, &o->sv_vNPol, &o->sv_codNC, &o->sv_compNC, &o->sv_bNTor, &o->sv_bNPol})
    c->init(o->N, o->H);
  if (o->Nic > 1)
    for (Coll* c : {&o->icTor, &o->icPol, &o->icNTor, &o->icNPol, &o->sv_icNTor, &o->sv_icNPol}) c->init(o->Nic, o->H);
  {  // rot_precompute (rotation.F90:20-33): 8 pi / 15 r_i^5
    const double ri = o->oc.R(1, 1), r2 = ri * ri, r4 = r2 * r2;
    o->rot_inertia = (8.0 * d_PI / 15.0) * (r4 * ri);
  }
  if (build_matrices(*o)) { *status = LSD_ESINGULAR; delete o; return nullptr; }
  return o;
}
void orc_destroy(Oracle* o) { delete o; }
// io_load_radial_txtfiles (io.F90:559-608): prof = the seven columns of
// planet_model.txt.in, [7][N]: rho, xi = rho'/rho, dxi/dr, T, dT/dr, eta, deta/dr.
// Rebuilds the radial mesh weights/bands and the operators (mes_precompute + *_matrices).
int orc_set_reference_state(Oracle* o, const double* prof) {
  if (o->cfg.boussinesq) return LSD_EARG;
  RDom& D = o->oc;
  const int N = o->N;
  std::vector<double>* cols[7] = {&D.rho0, &D.rho1, &D.rho2, &D.temp0, &D.temp1, &D.eta0, &D.eta1};
  for (int k = 0; k < 7; ++k) cols[k]->assign(prof + (size_t)k * N, prof + (size_t)(k + 1) * N);
  if (rdom_init(D, o->KL)) return LSD_ESINGULAR;
  if (build_matrices(*o)) return LSD_ESINGULAR;
  return 0;
}
void orc_sizes(const Oracle* o, lsd_sizes* s) {
  s->H = o->H; s->Th = o->Th; s->Th2 = o->Th2; s->Ph = o->Ph; s->Ma = o->Ma; s->Hc = o->Hc; s->Hr = o->Hr;
  s->N = o->N; s->L = o->L; s->M = o->M; s->Mp = o->Mp; s->KL = o->KL;
}
void orc_harmonics(const Oracle* o, int* l, int* m, int* s) {
  for (int i = 0; i < o->H; ++i) { l[i] = o->hl[i]; m[i] = o->hm[i]; s[i] = o->hs[i]; }
}
void orc_theta_map(const Oracle* o, int* thm) { for (int i = 0; i < 2 * o->Hc; ++i) thm[i] = o->thm[i]; }
void orc_radial_grid(const Oracle* o, double* r) { for (int n = 0; n < o->N; ++n) r[n] = o->oc.R(n + 1, 1); }
void orc_radial_weights(const Oracle* o, double* w) { for (int n = 0; n < o->N; ++n) w[n] = o->oc.intr2dr[n]; }
void orc_dr(const Oracle* o, int order, double* band) {  // (2KL+1, N)
  const Band& B = o->oc.dr[order];
  for (size_t i = 0; i < B.M.size(); ++i) band[i] = B.M[i];
}
void orc_gauss(const Oracle* o, double* gp, double* gw) { for (int j = 0; j < o->Th; ++j) { gp[j] = o->gp[j]; gw[j] = o->gw[j]; } }
int orc_legendre_table(const Oracle* o, int which, double* out) {
  const std::vector<double>* t = nullptr;
  switch (which) {
    case LSD_LEG_P: t = &o->P; break;
    case LSD_LEG_P_: t = &o->P_; break;
    case LSD_LEG_SIN1MP: t = &o->sin1mP; break;
    case LSD_LEG_LLP_: t = &o->llP_; break;
    case LSD_LEG_LLSIN1MP: t = &o->llsin1mP; break;
    case LSD_LEG_GWP: t = &o->gwP; break;
    case LSD_LEG_GWLLP_: t = &o->gwllP_; break;
    case LSD_LEG_GWLLSIN1MP: t = &o->gwllsin1mP; break;
    default: return LSD_EARG;
  }
  std::memcpy(out, t->data(), t->size() * sizeof(double));
  return 0;
}
// The operators applied to right-hand sides the way lsd_operator_solve_device does:
// tim_zerobc + tim_invX (timestep.F90:566-588) with the field's operator, the poloidal
// velocity as XGre, XPol and vel_gre_adjust (velocity.F90:369-395, 445-465, no Y multiply).
// re, im: (H, N) C order, in place.
int orc_operator_solve(Oracle* o, int field, double* re, double* im) {
  Coll b;
  b.init(o->N, o->H);
  std::memcpy(b.re.data(), re, b.re.size() * 8);
  std::memcpy(b.im.data(), im, b.im.size() * 8);
  tim_zerobc(*o, b);
  switch (field) {
    case LSD_VEL_TOR: tim_invX(*o, false, o->XTor, b); break;
    case LSD_VEL_POL:
      tim_invX(*o, false, o->XGre, b);
      tim_zerobc(*o, b);
      tim_invX(*o, false, o->XPol, b);
      vel_gre_adjust(*o, b);
      break;
    case LSD_COD_C: tim_invX(*o, true, o->XC, b); break;
    case LSD_COMP_C: tim_invX(*o, true, o->XComp, b); break;
    case LSD_MAG_TOR: if (o->Nic > 1) return LSD_EARG; tim_invX(*o, false, o->mXTor, b); break;
    case LSD_MAG_POL: if (o->Nic > 1) return LSD_EARG; tim_invX(*o, false, o->mXPol, b); break;
    default: return LSD_EARG;
  }
  std::memcpy(re, b.re.data(), b.re.size() * 8);
  std::memcpy(im, b.im.data(), b.im.size() * 8);
  return 0;
}
// LU factors of one operator: which 0 XTor 1 XPol 2 XGre 3 XC 4 mXTor 5 mXPol
int orc_operator_lu(const Oracle* o, int which, int l, double* ab, int* ipiv) {
  const std::vector<LUBand>* v[] = {&o->XTor, &o->XPol, &o->XGre, &o->XC, &o->mXTor, &o->mXPol};
  if (which < 0 || which > 5 || l < 0 || l >= o->L) return LSD_EARG;
  const LUBand& A = (*v[which])[l];
  if (A.M.empty()) return LSD_EARG;
  std::memcpy(ab, A.M.data(), A.M.size() * sizeof(double));
  for (int i = 0; i < A.N; ++i) ipiv[i] = A.ipiv[i];
  return 0;
}
// LAPACK restatements exposed for pinning against scipy
int orc_dgbtrf(int n, int kl, double* ab, int* ipiv) { return dgbtf2(n, kl, kl, ab, 3 * kl + 1, ipiv); }
void orc_dgbtrs(int n, int kl, const double* ab, const int* ipiv, double* b) { dgbtrs1(n, kl, kl, ab, 3 * kl + 1, ipiv, b); }
int orc_mat_invert(int n, double* a) { return mat_invert(n, a, n); }
// FFT restatement exposed for pinning against numpy: c2r of Y(0:Ma) -> x(0:Ph-1)
void orc_fft_c2r(int n, const double* yre, const double* yim, int nbins, double* x) {
  FFTPlan p; p.init(n);
  std::vector<cplx> a(n, 0.0), b(n), s(n);
  for (int k = 0; k < nbins && k <= n / 2; ++k) {
    if (k == 0 || 2 * k == n) a[k] = yre[k];
    else { a[k] = cplx(yre[k], yim[k]); a[n - k] = cplx(yre[k], -yim[k]); }
  }
  p.exec(a.data(), b.data(), +1, s.data());
  for (int i = 0; i < n; ++i) x[i] = b[i].real();
}
void orc_fft_r2c(int n, const double* x, double* yre, double* yim) {
  FFTPlan p; p.init(n);
  std::vector<cplx> a(n), b(n), s(n);
  for (int i = 0; i < n; ++i) a[i] = x[i];
  p.exec(a.data(), b.data(), -1, s.data());
  for (int k = 0; k <= n / 2; ++k) { yre[k] = b[k].real(); yim[k] = (k == 0 || 2 * k == n) ? 0.0 : b[k].imag(); }
}

int orc_set_rotation(Oracle* o, double omega) { o->rot_omega = omega; return 0; }
void orc_get_rotation(const Oracle* o, double* out) {
  out[0] = o->rot_omega; out[1] = o->rot_velTorq; out[2] = o->rot_magTorq;
}
int orc_set_coll(Oracle* o, int f, const double* re, const double* im) {
  Coll* c = field_ptr(*o, f);
  if (!c) return LSD_EARG;
  std::memcpy(c->re.data(), re, c->re.size() * sizeof(double));
  std::memcpy(c->im.data(), im, c->im.size() * sizeof(double));
  if (f == LSD_MAG_TOR || f == LSD_MAG_POL) {  // io_ic_extend with Ni = 1: ic = oc at r_i
    Coll& ic = f == LSD_MAG_TOR ? o->bicTor : o->bicPol;
    for (int nh = 0; nh < o->H; ++nh) { ic.re[(size_t)o->N * nh] = re[(size_t)o->N * nh]; ic.im[(size_t)o->N * nh] = im[(size_t)o->N * nh]; }
  }
  return 0;
}
int orc_get_coll(Oracle* o, int f, double* re, double* im) {
  Coll* c = field_ptr(*o, f);
  if (!c) return LSD_EARG;
  std::memcpy(re, c->re.data(), c->re.size() * sizeof(double));
  std::memcpy(im, c->im.data(), c->im.size() * sizeof(double));
  return 0;
}
int orc_get_nonlinear(Oracle* o, int f, double* re, double* im) {
  Coll* c = nl_ptr(*o, f);
  if (!c) return LSD_EARG;
  std::memcpy(re, c->re.data(), c->re.size() * sizeof(double));
  std::memcpy(im, c->im.data(), c->im.size() * sizeof(double));
  return 0;
}
void orc_set_time(Oracle* o, double t) { o->tim_t = t; }
// io_load_state's tim_dt (io.F90:426-429) with the matrices at that dt
int orc_set_dt(Oracle* o, double dt) {
  if (!(dt > 0)) return LSD_EARG;
  o->tim_dt = dt;
  return build_matrices(*o) ? LSD_ESINGULAR : 0;
}
void orc_dt_control(const Oracle* o, double* out) { out[0] = o->tim_dt; out[1] = o->tim_corr_dt; out[2] = o->tim_cfl_dt; }

int orc_spec2phys(Oracle* o, const double* sre, const double* sim, double* p) {
  Spec s; s.init(o->N, o->H);
  std::memcpy(s.re.data(), sre, s.re.size() * 8); std::memcpy(s.im.data(), sim, s.im.size() * 8);
  Phys x; tra_spec2phys(*o, s, x);
  std::memcpy(p, x.data(), x.size() * 8);
  return 0;
}
int orc_phys2spec(Oracle* o, const double* p, double* sre, double* sim) {
  Phys x((size_t)o->Th * o->Ph * o->N);
  std::memcpy(x.data(), p, x.size() * 8);
  Spec s; tra_phys2spec(*o, x, s);
  std::memcpy(sre, s.re.data(), s.re.size() * 8); std::memcpy(sim, s.im.data(), s.im.size() * 8);
  return 0;
}
int orc_qst2rtp(Oracle* o, const double* qr, const double* qi, const double* sr, const double* si,
                const double* tr, const double* ti, double* r, double* th, double* ph) {
  Spec q, s, t;
  q.init(o->N, o->H); s.init(o->N, o->H); t.init(o->N, o->H);
  size_t n = q.re.size() * 8;
  std::memcpy(q.re.data(), qr, n); std::memcpy(q.im.data(), qi, n);
  std::memcpy(s.re.data(), sr, n); std::memcpy(s.im.data(), si, n);
  std::memcpy(t.re.data(), tr, n); std::memcpy(t.im.data(), ti, n);
  Phys a, b, c; tra_qst2rtp(*o, q, s, t, a, b, c);
  size_t pn = a.size() * 8;
  std::memcpy(r, a.data(), pn); std::memcpy(th, b.data(), pn); std::memcpy(ph, c.data(), pn);
  return 0;
}
int orc_qst2rtp_vel(Oracle* o, const double* const* in /*12: q s t qr sr tr, re/im*/, double* const* out /*8*/) {
  Spec sp[6];
  size_t n = (size_t)o->N * o->H * 8;
  for (int k = 0; k < 6; ++k) {
    sp[k].init(o->N, o->H);
    std::memcpy(sp[k].re.data(), in[2 * k], n); std::memcpy(sp[k].im.data(), in[2 * k + 1], n);
  }
  Phys ph[8];
  Phys* outs[8];
  for (int k = 0; k < 8; ++k) outs[k] = &ph[k];
  tra_qst2rtp_vel(*o, sp[0], sp[1], sp[2], sp[3], sp[4], sp[5], outs);
  for (int k = 0; k < 8; ++k) std::memcpy(out[k], ph[k].data(), ph[k].size() * 8);
  return 0;
}
int orc_rtp2qst(Oracle* o, const double* r, const double* th, const double* ph, double* qr, double* qi,
                double* sr, double* si, double* tr, double* ti) {
  size_t psz = (size_t)o->Th * o->Ph * o->N;
  Phys a(psz), b(psz), c(psz);
  std::memcpy(a.data(), r, psz * 8); std::memcpy(b.data(), th, psz * 8); std::memcpy(c.data(), ph, psz * 8);
  Spec q, s, t; tra_rtp2qst(*o, a, b, c, q, s, t);
  size_t n = q.re.size() * 8;
  std::memcpy(qr, q.re.data(), n); std::memcpy(qi, q.im.data(), n);
  std::memcpy(sr, s.re.data(), n); std::memcpy(si, s.im.data(), n);
  std::memcpy(tr, t.re.data(), n); std::memcpy(ti, t.im.data(), n);
  return 0;
}
int orc_grad(Oracle* o, const double* sre, const double* sim, double* th, double* ph) {
  Spec s; s.init(o->N, o->H);
  std::memcpy(s.re.data(), sre, s.re.size() * 8); std::memcpy(s.im.data(), sim, s.im.size() * 8);
  Phys a, b; tra_grad(*o, s, a, b);
  std::memcpy(th, a.data(), a.size() * 8); std::memcpy(ph, b.data(), b.size() * 8);
  return 0;
}

int orc_dth(Oracle* o, const double* sre, const double* sim, double* p) {
  Spec s; s.init(o->N, o->H);
  std::memcpy(s.re.data(), sre, s.re.size() * 8); std::memcpy(s.im.data(), sim, s.im.size() * 8);
  Phys a; tra_dth(*o, s, a);
  std::memcpy(p, a.data(), a.size() * 8);
  return 0;
}
int orc_nonlinear(Oracle* o) { evaluate(*o); return 0; }
int orc_predictor(Oracle* o) { predictor(*o); o->tim_it = 1; return 0; }
int orc_corrector(Oracle* o, double* dterr) {
  corrector(*o);
  if (dterr) *dterr = o->tim_dterr;
  return 0;
}
// main loop (main.F90:100-164) for nsteps completed steps; fixed dt
int orc_step(Oracle* o, int nsteps, lsd_stats* st) {
  int done = 0, corr = 0, evals = 0;
  double last = 0;
  while (done < nsteps) {
    evaluate(*o); ++evals;
    if (o->tim_it == 0) {
      if (o->cfg.timestep < 0) {  // main.F90:126-134
        non_maxtstep(*o);
        tim_new_tstep(*o);
        if (o->tim_new_dt && build_matrices(*o)) return LSD_ESINGULAR;
      }
      predictor(*o);
      o->tim_it = 1;
    } else {
      corrector(*o); ++corr;
      last = o->tim_dterr;
      if (check_cgce(*o)) return LSD_ENOTCONVERGED;
    }
    if (o->tim_it == 0) {
      o->tim_t = o->tim_t + o->tim_dt;
      o->tim_step = o->tim_step + 1;
      ++done;
    }
  }
  if (st) {
    st->steps_done = done; st->correctors = corr; st->evaluations = evals; st->kernel_launches = 0;
    st->last_dterr = last; st->t = o->tim_t; st->dt = o->tim_dt;
  }
  return 0;
}
// tim_check_cgce / tim_new_tstep on a bare loop state (lsd_pc_state), for the
// comparison with the library's C-ABI mirrors
struct TimOnly {
  lsd_config cfg;
  double tim_t, tim_dt, tim_dterr, tim_corr_dt, tim_cfl_dt, lasterr;
  int tim_it, tim_step, tim_pcn;
  bool tim_new_dt;
};
static TimOnly tim_in(const lsd_config* cfg, const lsd_pc_state* s) {
  TimOnly o;
  o.cfg = *cfg;
  o.tim_t = s->t; o.tim_dt = s->dt; o.tim_dterr = s->dterr; o.tim_corr_dt = s->corr_dt; o.lasterr = s->lasterr;
  o.tim_cfl_dt = s->cfl_dt; o.tim_it = s->it; o.tim_step = s->step; o.tim_pcn = s->pcn; o.tim_new_dt = false;
  return o;
}
static void tim_out(const TimOnly& o, lsd_pc_state* s) {
  s->t = o.tim_t; s->dt = o.tim_dt; s->dterr = o.tim_dterr; s->corr_dt = o.tim_corr_dt; s->lasterr = o.lasterr;
  s->cfl_dt = o.tim_cfl_dt; s->it = o.tim_it; s->step = o.tim_step; s->pcn = o.tim_pcn;
}
int orc_tim_check_cgce(const lsd_config* cfg, lsd_pc_state* s) {
  TimOnly o = tim_in(cfg, s);
  const int fail = check_cgce(o);
  tim_out(o, s);
  return fail ? LSD_ENOTCONVERGED : 0;
}
int orc_tim_new_tstep(const lsd_config* cfg, lsd_pc_state* s, int* new_dt) {
  TimOnly o = tim_in(cfg, s);
  tim_new_tstep(o);
  tim_out(o, s);
  *new_dt = o.tim_new_dt ? 1 : 0;
  return 0;
}
int orc_energies(Oracle* o, double* out) { energies(*o, out); return 0; }
int orc_diagnostics(Oracle* o, double* scalars, double* spectra, double* profiles) {
  diagnostics(*o, scalars, spectra, profiles);
  return 0;
}

}  // extern "C"
