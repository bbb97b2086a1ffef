// lsd_banded.cuh -- FP64 banded LU (partial pivoting) and small dense inverses, device side.
//
// Same algorithms as LAPACK's unblocked dgbtf2 / dgbtrs (with dtbsv) and dgetf2 / dgetri
// (with dtrti2), which the reference calls through mes_lu_find (meshs.F90:447-456),
// tim_invX (timestep.F90:566-588) and mes_mat_invert (meshs.F90:427-440).  Band storage
// is LAPACK's: A(i,j) at ab[(kl+ku+i-j) + ldab*(j-1)] (1-based i,j), ldab = 2kl+ku+1.
#pragma once
#include "lsd_common.cuh"

// Factorise one n x n band matrix with kl = ku sub/super-diagonals in place.
// Returns 0 or the first zero-pivot column (LAPACK info).
__device__ inline int dev_dgbtf2(int n, int kl, double* ab, int ldab, int* ipiv) {
  const int ku = kl, kv = ku + kl;
#define AB(i, j) ab[(size_t)((i) - 1) + (size_t)ldab * ((j) - 1)]
  int info = 0;
  for (int j = ku + 2; j <= min(kv, n); ++j)
    for (int i = kv - j + 2; i <= kl; ++i) AB(i, j) = 0.0;
  int ju = 1;
  for (int j = 1; j <= n; ++j) {
    if (j + kv <= n)
      for (int i = 1; i <= kl; ++i) AB(i, j + kv) = 0.0;
    int km = min(kl, n - j);
    int jp = 1;
    double amax = fabs(AB(kv + 1, j));
    for (int i = 2; i <= km + 1; ++i) {
      double v = fabs(AB(kv + i, j));
      if (v > amax) { amax = v; jp = i; }
    }
    ipiv[j - 1] = jp + j - 1;
    if (AB(kv + jp, j) != 0.0) {
      ju = max(ju, min(j + ku + jp - 1, n));
      if (jp != 1) {
        for (int c = 0; c <= ju - j; ++c) {
          double t = AB(kv + jp - c, j + c);
          AB(kv + jp - c, j + c) = AB(kv + 1 - c, j + c);
          AB(kv + 1 - c, j + c) = t;
        }
      }
      if (km > 0) {
        double rp = 1.0 / AB(kv + 1, j);
        for (int i = 1; i <= km; ++i) AB(kv + 1 + i, j) *= rp;
        if (ju > j) {
          for (int c = 1; c <= ju - j; ++c) {
            double y = AB(kv + 1 - c, j + c);
            if (y != 0.0) {
              double temp = -y;
              for (int i = 1; i <= km; ++i)
                AB(kv + 1 - c + i, j + c) = AB(kv + 1 - c + i, j + c) + AB(kv + 1 + i, j) * temp;
            }
          }
        }
      }
    } else if (info == 0) {
      info = j;
    }
  }
#undef AB
  return info;
}

// Solve with the factors of dev_dgbtf2 for one right-hand side (dgbtrs 'N').
__device__ inline void dev_dgbtrs1(int n, int kl, const double* ab, int ldab, const int* ipiv,
                                   double* b) {
  const int ku = kl, kd = ku + kl + 1;
#define AB(i, j) ab[(size_t)((i) - 1) + (size_t)ldab * ((j) - 1)]
  for (int j = 1; j <= n - 1; ++j) {
    int lm = min(kl, n - j);
    int l = ipiv[j - 1];
    if (l != j) { double t = b[l - 1]; b[l - 1] = b[j - 1]; b[j - 1] = t; }
    double y = b[j - 1];
    if (y != 0.0) {
      double temp = -y;
      for (int i = 1; i <= lm; ++i) b[j + i - 1] = b[j + i - 1] + AB(kd + i, j) * temp;
    }
  }
  const int k = kl + ku, kplus1 = k + 1;
  for (int j = n; j >= 1; --j) {
    if (b[j - 1] != 0.0) {
      int l = kplus1 - j;
      b[j - 1] = b[j - 1] / AB(kplus1, j);
      double temp = b[j - 1];
      for (int i = j - 1; i >= max(1, j - k); --i) b[i - 1] = b[i - 1] - temp * AB(l + i, j);
    }
  }
#undef AB
}

// In-place inverse of a small dense matrix (lda >= n), dgetf2 + dtrti2 + dgetri order.
__device__ inline int dev_mat_invert(int n, double* a, int lda) {
#define A_(i, j) a[(size_t)((i) - 1) + (size_t)lda * ((j) - 1)]
  int ipiv[2 * LSD_MAX_KL + 1];
  double work[2 * LSD_MAX_KL + 1];
  const double sfmin = 2.2250738585072014e-308;
  for (int j = 1; j <= n; ++j) {
    int jp = j;
    double amax = fabs(A_(j, j));
    for (int i = j + 1; i <= n; ++i)
      if (fabs(A_(i, j)) > amax) { amax = fabs(A_(i, j)); jp = i; }
    ipiv[j - 1] = jp;
    if (A_(jp, j) == 0.0) return j;
    if (jp != j)
      for (int c = 1; c <= n; ++c) { double t = A_(j, c); A_(j, c) = A_(jp, c); A_(jp, c) = t; }
    if (j < n) {
      if (fabs(A_(j, j)) >= sfmin) {
        double r = 1.0 / A_(j, j);
        for (int i = j + 1; i <= n; ++i) A_(i, j) *= r;
      } else {
        for (int i = j + 1; i <= n; ++i) A_(i, j) = A_(i, j) / A_(j, j);
      }
      for (int c = j + 1; c <= n; ++c) {
        double y = A_(j, c);
        if (y != 0.0) {
          double temp = -y;
          for (int i = j + 1; i <= n; ++i) A_(i, c) = A_(i, c) + A_(i, j) * temp;
        }
      }
    }
  }
  for (int j = 1; j <= n; ++j) {
    A_(j, j) = 1.0 / A_(j, j);
    double ajj = -A_(j, j);
    for (int jj = 1; jj <= j - 1; ++jj) {
      double x = A_(jj, j);
      if (x != 0.0) {
        double temp = x;
        for (int i = 1; i <= jj - 1; ++i) A_(i, j) = A_(i, j) + temp * A_(i, jj);
        A_(jj, j) *= A_(jj, jj);
      }
    }
    for (int i = 1; i <= j - 1; ++i) A_(i, j) *= ajj;
  }
  for (int j = n; j >= 1; --j) {
    for (int i = j + 1; i <= n; ++i) { work[i - 1] = A_(i, j); A_(i, j) = 0.0; }
    if (j < n) {
      for (int c = j + 1; c <= n; ++c) {
        double temp = -work[c - 1];
        if (work[c - 1] != 0.0)
          for (int i = 1; i <= n; ++i) A_(i, j) = A_(i, j) + temp * A_(i, c);
      }
    }
  }
  for (int j = n - 1; j >= 1; --j) {
    int jp = ipiv[j - 1];
    if (jp != j)
      for (int i = 1; i <= n; ++i) { double t = A_(i, j); A_(i, j) = A_(i, jp); A_(i, jp) = t; }
  }
#undef A_
  return 0;
}
