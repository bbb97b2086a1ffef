// lsd_fft.cu -- batched real FFTs in phi, standalone and fused with the physical-space
// nonlinear products.
//
// Contract restated from the reference's FFTW use (transform.fftw3.F90:78-93, 280-466):
//  * synthesis (c2r, unnormalised): bins 0..M-1 come from the m-counter map var_Th%m,
//    bins M..Ph/2 are zero, the imaginary part of bin 0 is ignored;
//  * analysis (r2c): input scaled by 1/Ph first, bins 0..M-1 kept, bin 0 exactly real.
// A real row of length Ph = 2 P2 is transformed as one complex FFT of length P2 of the
// interleaved samples z[t] = x[2t] + i x[2t+1], with the usual split pre-/post-processing.
//
// Each complex FFT of length P2 = E G (G a power of two <= 16) is two shared-memory
// passes of in-register DFTs (the "four-step" split k = k1 + G k2, t = t1 + E t2):
//   column pass: G threads per row, an E-point DFT over k2 and the twiddle w^(t1 k1);
//   row pass:    E threads per row, a G-point DFT over k1.
// Rows are padded by one complex per G values, so both passes read and write shared
// memory without bank conflicts.  The inverse leaves the samples transposed (position
// (G+1) t1 + t2 holds x[t1 + E t2]); the forward transform is the mirror image, takes
// them back in that order and returns the spectrum in natural order, so the point-wise
// products never need a reordering.
//
// The theta-Fourier rows are stored in half-row pairs ([n][h/2][m-counter][E/O][h%2],
// four_off); one CTA of the fused kernel owns one pair (four full theta rows: the
// southern and northern row of each half-row), reads the 15 synthesised fields of u,
// curl u, B, curl B and grad C as contiguous 8 KB blocks, transforms them, forms
//   u x (curl u) + Coriolis + Lorentz      (nonlinear.F90:70-146, Boussinesq)
//   -(Pr/Pm) u . grad C                     (nonlinear.F90:269-272)
//   u x B                                   (nonlinear.F90:421-430)
// at every grid point in shared memory, transforms the 7 results back and writes their
// folded theta-Fourier rows in the analysis layout (four_off_a).  Physical-space fields
// never touch HBM.
#include <algorithm>
#include <type_traits>

#include "lsd_common.cuh"

namespace {

struct FFTPlanDev {
  int P2, Ph, M, NM, Th, Th2, HB, Mp;
  const double2* tw2;  // e^{+2 pi i k/P2}, k < P2
  const double2* twh;  // e^{+2 pi i k/Ph}, k < Ph
  const int* thm;      // m-counter -> bin
  const int* bin2c;    // bin -> m-counter (M entries)
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 add2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 sub2(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// In-register DFT of length N (mixed radix 2/3, decimation in time) with the twiddles of
// the full length EF: w[j] = e^{+2 pi i j / EF} (a shared-memory table, read as
// broadcasts); SIGN +1 inverse, -1 forward.
template <int SIGN>
__device__ __forceinline__ double2 twid(double2 a, double2 w) { return SIGN > 0 ? cmul(a, w) : cmulc(a, w); }

// Short DFTs with their constants written out (no twiddle tables): 3- and 4-point
// butterflies, 16 = 4 x 4 (radix 4 with the 16th roots of unity), and the prime-factor
// (Good-Thomas) splits 6 = 2 x 3 and 12 = 3 x 4, which need no twiddles at all: input
// index n = (N2 n1 + N1 n2) mod N, output index k = (N2 <N2^-1>_N1 k1 + N1 <N1^-1>_N2 k2) mod N.
constexpr double kSqrt3_2 = 0.86602540378443864676;  // sin(pi/3)
constexpr double kSqrt2_2 = 0.70710678118654752440;  // cos(pi/4)
constexpr double kCos8 = 0.92387953251128675613;     // cos(pi/8)
constexpr double kSin8 = 0.38268343236508977173;     // sin(pi/8)

template <int SIGN>
__device__ __forceinline__ double2 mul_i(double2 a) {  // a * (SIGN i)
  return SIGN > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}
template <int SIGN>
__device__ __forceinline__ void dft3(double2& a, double2& b, double2& c) {
  const double2 t1 = add2(b, c);
  const double2 t2 = make_double2(a.x - 0.5 * t1.x, a.y - 0.5 * t1.y);
  const double2 t3 = make_double2(SIGN * kSqrt3_2 * (b.x - c.x), SIGN * kSqrt3_2 * (b.y - c.y));
  a = add2(a, t1);
  b = make_double2(t2.x - t3.y, t2.y + t3.x);
  c = make_double2(t2.x + t3.y, t2.y - t3.x);
}
template <int SIGN>
__device__ __forceinline__ void dft4(double2& x0, double2& x1, double2& x2, double2& x3) {
  const double2 a = add2(x0, x2), b = sub2(x0, x2), c = add2(x1, x3), d = mul_i<SIGN>(sub2(x1, x3));
  x0 = add2(a, c);
  x1 = add2(b, d);
  x2 = sub2(a, c);
  x3 = sub2(b, d);
}
// multiplication by w16^e, w16 = e^{SIGN 2 pi i / 16}, e in {1, 2, 3, 6, 9}
template <int SIGN, int E16>
__device__ __forceinline__ double2 tw16(double2 a) {
  double c, s;
  if (E16 == 1) { c = kCos8; s = kSin8; }
  else if (E16 == 2) { c = kSqrt2_2; s = kSqrt2_2; }
  else if (E16 == 3) { c = kSin8; s = kCos8; }
  else if (E16 == 6) { c = -kSqrt2_2; s = kSqrt2_2; }
  else { c = -kCos8; s = -kSin8; }  // 9
  s = SIGN * s;
  return make_double2(a.x * c - a.y * s, a.x * s + a.y * c);
}
template <int SIGN>
__device__ __forceinline__ void dft16(double2 (&x)[16]) {
  // columns n2: 4-point DFTs over n1 of x[4 n1 + n2], then the twiddles w16^(n2 k1)
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) dft4<SIGN>(x[n2], x[4 + n2], x[8 + n2], x[12 + n2]);
  // x[4 k1 + n2] now holds Y[n2][k1]
  x[4 * 1 + 1] = tw16<SIGN, 1>(x[4 * 1 + 1]);
  x[4 * 2 + 1] = tw16<SIGN, 2>(x[4 * 2 + 1]);
  x[4 * 3 + 1] = tw16<SIGN, 3>(x[4 * 3 + 1]);
  x[4 * 1 + 2] = tw16<SIGN, 2>(x[4 * 1 + 2]);
  x[4 * 2 + 2] = mul_i<SIGN>(x[4 * 2 + 2]);
  x[4 * 3 + 2] = tw16<SIGN, 6>(x[4 * 3 + 2]);
  x[4 * 1 + 3] = tw16<SIGN, 3>(x[4 * 1 + 3]);
  x[4 * 2 + 3] = tw16<SIGN, 6>(x[4 * 2 + 3]);
  x[4 * 3 + 3] = tw16<SIGN, 9>(x[4 * 3 + 3]);
  // rows k1: 4-point DFTs over n2 give X[k1 + 4 k2]
  double2 y[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    double2 a = x[4 * k1], b = x[4 * k1 + 1], c = x[4 * k1 + 2], d = x[4 * k1 + 3];
    dft4<SIGN>(a, b, c, d);
    y[k1] = a; y[k1 + 4] = b; y[k1 + 8] = c; y[k1 + 12] = d;
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) x[i] = y[i];
}
template <int SIGN>
__device__ __forceinline__ void dft12(double2 (&x)[12]) {  // 3 x 4, n = (4 n1 + 3 n2) % 12
  double2 y[3][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    double2 a = x[(3 * n2) % 12], b = x[(4 + 3 * n2) % 12], c = x[(8 + 3 * n2) % 12];
    dft3<SIGN>(a, b, c);
    y[0][n2] = a; y[1][n2] = b; y[2][n2] = c;
  }
#pragma unroll
  for (int k1 = 0; k1 < 3; ++k1) {
    dft4<SIGN>(y[k1][0], y[k1][1], y[k1][2], y[k1][3]);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) x[(4 * k1 + 9 * k2) % 12] = y[k1][k2];
  }
}
template <int SIGN>
__device__ __forceinline__ void dft6(double2 (&x)[6]) {  // 2 x 3, n = (3 n1 + 2 n2) % 6
  double2 y[2][3];
#pragma unroll
  for (int n2 = 0; n2 < 3; ++n2) {
    const double2 a = x[(2 * n2) % 6], b = x[(3 + 2 * n2) % 6];
    y[0][n2] = add2(a, b);
    y[1][n2] = sub2(a, b);
  }
#pragma unroll
  for (int k1 = 0; k1 < 2; ++k1) {
    dft3<SIGN>(y[k1][0], y[k1][1], y[k1][2]);
#pragma unroll
    for (int k2 = 0; k2 < 3; ++k2) x[(3 * k1 + 4 * k2) % 6] = y[k1][k2];
  }
}

template <int N, int EF, int SIGN>
__device__ __forceinline__ void rdft(double2 (&x)[N], const double2* w) {
  if constexpr (N == 1) {
    return;
  } else if constexpr (N == 16) {
    dft16<SIGN>(x);
  } else if constexpr (N == 12) {
    dft12<SIGN>(x);
  } else if constexpr (N == 6) {
    dft6<SIGN>(x);
  } else if constexpr (N == 4) {
    dft4<SIGN>(x[0], x[1], x[2], x[3]);
  } else if constexpr (N == 2) {
    const double2 a = x[0], b = x[1];
    x[0] = add2(a, b);
    x[1] = sub2(a, b);
  } else if constexpr (N == 3) {
    const double h = 0.86602540378443864676;  // sqrt(3)/2
    const double2 a = x[0], b = x[1], c = x[2];
    const double2 t1 = add2(b, c);
    const double2 t2 = make_double2(a.x - 0.5 * t1.x, a.y - 0.5 * t1.y);
    const double2 t3 = make_double2(SIGN * h * (b.x - c.x), SIGN * h * (b.y - c.y));
    x[0] = add2(a, t1);
    x[1] = make_double2(t2.x - t3.y, t2.y + t3.x);  // t2 + i t3
    x[2] = make_double2(t2.x + t3.y, t2.y - t3.x);  // t2 - i t3
  } else if constexpr (N % 2 == 0) {
    constexpr int H = N / 2;
    double2 ev[H], od[H];
#pragma unroll
    for (int i = 0; i < H; ++i) { ev[i] = x[2 * i]; od[i] = x[2 * i + 1]; }
    rdft<H, EF, SIGN>(ev, w);
    rdft<H, EF, SIGN>(od, w);
#pragma unroll
    for (int k = 0; k < H; ++k) {
      const double2 t = k ? twid<SIGN>(od[k], w[k * (EF / N)]) : od[0];
      x[k] = add2(ev[k], t);
      x[k + H] = sub2(ev[k], t);
    }
  } else {
    static_assert(N % 3 == 0, "DFT length must be 2^a 3^b");
    constexpr int T = N / 3;
    double2 s0[T], s1[T], s2[T];
#pragma unroll
    for (int i = 0; i < T; ++i) { s0[i] = x[3 * i]; s1[i] = x[3 * i + 1]; s2[i] = x[3 * i + 2]; }
    rdft<T, EF, SIGN>(s0, w);
    rdft<T, EF, SIGN>(s1, w);
    rdft<T, EF, SIGN>(s2, w);
#pragma unroll
    for (int k = 0; k < T; ++k) {
      double2 y[3] = {s0[k], k ? twid<SIGN>(s1[k], w[k * (EF / N)]) : s1[0],
                      k ? twid<SIGN>(s2[k], w[(2 * k * (EF / N)) % EF]) : s2[0]};
      rdft<3, EF, SIGN>(y, w);
      x[k] = y[0];
      x[k + T] = y[1];
      x[k + 2 * T] = y[2];
    }
  }
}

// Per-CTA shared tables of one transform length P2 = E G:
//   tw[t1 G + k1] = e^{+2 pi i t1 k1 / P2}   column-pass twiddles (read by consecutive k1)
//   twE[j] = e^{+2 pi i j / E},  twG[j] = e^{+2 pi i j / G}   register-DFT twiddles
//   twh[k] = e^{+2 pi i k / Ph}, k < P2      real-FFT packing / unpacking twiddles
//   thm[c] = FFT bin of m-counter c,  b2c[b] = m-counter of bin b < M
// (in shared memory, so that no load of the packing, gathering or unpacking waits on
// another global load)
struct FFTTabs {
  double2* tw;
  double2* twE;
  double2* twG;
  double2* twh;
  int* thm;
  int* b2c;
};

__host__ __device__ __forceinline__ size_t fft_tab_bytes(int P2, int E, int G, int NM) {
  return sizeof(double2) * (2 * (size_t)P2 + E + G) + sizeof(int) * (size_t)(((NM + 3) & ~3) + ((P2 + 3) & ~3));
}

// carve the tables out of `base` (16-byte aligned) and fill them; ends with a barrier
template <int E, int G>
__device__ __forceinline__ FFTTabs fft_tabs_init(unsigned char* base, const FFTPlanDev& pl) {
  FFTTabs t;
  t.tw = (double2*)base;
  t.twE = t.tw + E * G;
  t.twG = t.twE + E;
  t.twh = t.twG + G;
  t.thm = (int*)(t.twh + E * G);
  t.b2c = t.thm + ((pl.NM + 3) & ~3);
  for (int i = threadIdx.x; i < E * G; i += blockDim.x) t.tw[i] = __ldg(&pl.tw2[(i / G) * (i % G)]);
  for (int i = threadIdx.x; i < E; i += blockDim.x) t.twE[i] = __ldg(&pl.tw2[G * i]);
  for (int i = threadIdx.x; i < G; i += blockDim.x) t.twG[i] = __ldg(&pl.tw2[E * i]);
  for (int i = threadIdx.x; i < E * G; i += blockDim.x) t.twh[i] = __ldg(&pl.twh[i]);
  for (int i = threadIdx.x; i < pl.NM; i += blockDim.x) t.thm[i] = __ldg(&pl.thm[i]);
  for (int i = threadIdx.x; i < pl.M; i += blockDim.x) t.b2c[i] = __ldg(&pl.bin2c[i]);
  __syncthreads();
  return t;
}

// padded position of natural index k (one pad slot after every G values)
template <int G>
__device__ __forceinline__ int ppos(int k) { return k + k / G; }

// Column pass over `nrows` rows of stride RS = E (G + 1).  SIGN +1 (inverse): E-point DFT
// over k2 of Z[k1 + G k2], then the twiddle w^(t1 k1).  SIGN -1 (forward): the twiddle
// w^(-t1 k1) first, then the E-point DFT.  In place.
template <int E, int G, int SIGN>
__device__ __forceinline__ void col_pass(double2* rows, int nrows, const FFTTabs& t) {
  constexpr int RS = E * (G + 1);
  for (int i = threadIdx.x; i < nrows * G; i += blockDim.x) {
    const int r = i / G, k1 = i - r * G;
    double2* col = rows + (size_t)r * RS + k1;
    double2 v[E];
#pragma unroll
    for (int k = 0; k < E; ++k) v[k] = col[k * (G + 1)];
    if (SIGN < 0) {
#pragma unroll
      for (int k = 1; k < E; ++k) v[k] = cmulc(v[k], t.tw[k * G + k1]);
    }
    rdft<E, E, SIGN>(v, t.twE);
    if (SIGN > 0) {
#pragma unroll
      for (int k = 1; k < E; ++k) v[k] = cmul(v[k], t.tw[k * G + k1]);
    }
#pragma unroll
    for (int k = 0; k < E; ++k) col[k * (G + 1)] = v[k];
  }
}

// Row pass: a G-point DFT over the G contiguous values of each (row, t1).  In place.
template <int E, int G, int SIGN>
__device__ __forceinline__ void row_pass(double2* rows, int nrows, const FFTTabs& t) {
  constexpr int RS = E * (G + 1);
  for (int i = threadIdx.x; i < nrows * E; i += blockDim.x) {
    const int r = i / E, t1 = i - r * E;
    double2* seg = rows + (size_t)r * RS + t1 * (G + 1);
    double2 v[G];
#pragma unroll
    for (int k = 0; k < G; ++k) v[k] = seg[k];
    rdft<G, G, SIGN>(v, t.twG);
#pragma unroll
    for (int k = 0; k < G; ++k) seg[k] = v[k];
  }
}

// Half-spectrum packing for the c2r: Z[k] from Y[k] and conj(Y[P2-k]) (Y[P2] = Nyquist = 0;
// the imaginary part of the DC bin is ignored).
__device__ __forceinline__ double2 c2r_pack(int k, double2 yk, double2 ymk, const double2* twh) {
  const double2 yc = conj2(ymk);
  if (k == 0) yk.y = 0.0;
  const double2 s = add2(yk, yc), d = sub2(yk, yc);
  const double2 wd = cmul(twh[k], d);
  return make_double2(s.x - wd.y, s.y + wd.x);  // s + i w d
}
// Bin k < P2 of the real spectrum from Z[k] and Z[P2-k] (Z[0] for k = 0).
__device__ __forceinline__ double2 r2c_unpack(int k, double2 zk, double2 zmk, const double2* twh) {
  if (k == 0) return make_double2(zk.x + zk.y, 0.0);
  const double2 zc = conj2(zmk);
  const double2 A = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
  const double2 Bi = make_double2(0.5 * (zk.x - zc.x), 0.5 * (zk.y - zc.y));  // i B
  const double2 B = make_double2(Bi.y, -Bi.x);
  return add2(A, cmulc(B, twh[k]));
}

// one 32-byte store of two complex values (p 32-byte aligned)
__device__ __forceinline__ void st_global_2c(cplx* p, double2 a, double2 b) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y)
               : "memory");
}

// theta row of half-row h on side 0 (south) / 1 (north)
__device__ __forceinline__ int row_theta(int h, int side, int Th) { return side ? Th - 1 - h : h; }

// A staged field: the folded rows of the CTA's half-row pair in bin order,
// sp[(p * 2 + jj) * M + b] (p = E/O).  Row (jj, side): Y = E + O (south), E - O (north);
// bins b >= M are zero.
__device__ __forceinline__ double2 row_bin(const double2* sp, int b, int jj, int side, int M) {
  if (b >= M) return make_double2(0.0, 0.0);
  const double2 e = sp[jj * M + b], o = sp[(2 + jj) * M + b];
  return side ? sub2(e, o) : add2(e, o);
}

// stage element i (raw order (c, p, jj)) of one field's (n, h/2) block into bin order
__device__ __forceinline__ void stage_elem(double2* sp, const cplx* blk, const FFTTabs& t, int M, int i) {
  const int c = i >> 2, p = (i >> 1) & 1, jj = i & 1;
  sp[(p * 2 + jj) * M + t.thm[c]] = blk[i];
}

// bin b < M of a transformed row (natural order, padded) as a real-spectrum bin
template <int G>
__device__ __forceinline__ double2 row_unpack(const double2* row, int b, int P2, const double2* twh) {
  return r2c_unpack(b, row[ppos<G>(b)], row[ppos<G>(b == 0 ? 0 : P2 - b)], twh);
}

// ---- fused: theta-Fourier inputs -> products -> theta-Fourier outputs ---------------------
// Product sets (the physical-space loops of nonlinear.F90):
//   PS_BOUSS       u, w = curl u, B, J = curl B, grad C (15)      -> u x w + Coriolis +
//                  Lorentz (3), u x B (3), -Pr/Pm u.grad C (1)      (:70-146, 269-272, 421-430)
//   PS_BOUSS_COMP  + grad Comp (18)                                  -> + -Sc/Pm u.grad Comp (8)
//   PS_ANEL_MOM    u, w, B, J (12) -> momentum with the compressible viscous force and
//                  the Lorentz force / rho (3), u x B (3)            (:70-146)
//   PS_ANEL_SCAL   u, w, J, grad C, dr u_r, dr u_th, dr u_ph (15) + qv1, qv2 (derived) ->
//                  entropy with dissipation (1)                      (:239-266)
//   PS_ANEL_SCAL_COMP  + grad Comp (18) -> + composition (2)         (:317-331)
// qv1 and qv2 (tra_qst2rtp_vel, transform.fftw3.F90:678-700) are not synthesised: with
// qva = m/sin llsin1mP - cot llP_ and qvb = cot llsin1mP - m/sin llP_ (legendre.F90:97-100)
// the Legendre sums collapse, per theta row and order m, to
//   qv1_m = (cot u_th,m + i m/sin u_ph,m) / r,   qv2_m = (i m/sin u_th,m - cot u_ph,m) / r,
// which are formed from the u_th, u_ph bins that the same CTA gathers.
enum ProdSet { PS_BOUSS = 0, PS_BOUSS_COMP, PS_ANEL_MOM, PS_ANEL_SCAL, PS_ANEL_SCAL_COMP };
template <int PS> struct PSet;
template <> struct PSet<PS_BOUSS> { static constexpr int in = 15, deriv = 0, out = 7; };
template <> struct PSet<PS_BOUSS_COMP> { static constexpr int in = 18, deriv = 0, out = 8; };
template <> struct PSet<PS_ANEL_MOM> { static constexpr int in = 12, deriv = 0, out = 6; };
template <> struct PSet<PS_ANEL_SCAL> { static constexpr int in = 15, deriv = 2, out = 1; };
template <> struct PSet<PS_ANEL_SCAL_COMP> { static constexpr int in = 18, deriv = 2, out = 2; };
constexpr int PROD_MAXIN = 18;

struct ProdConst {
  double d_Cor, Cmag, d_qm1, d_qm1c, Pm, E, Diss;
  const double* sn;   // sin(theta_j)
  const double* gp;   // cos(theta_j)
  const double* sn1;  // 1/sin(theta_j)
  const double* r;    // [7][N] powers of r
  const double* ref;  // [7][N] reference state (anelastic)
  unsigned long long* cflmax;  // variable dt: per-shell CFL maxima [N][2] (bits of doubles >= 0), or null
  double* rotsum;     // inner-core rotation: per half-row h the two torque surface sums of
                      // shell 0 at [2 h], [2 h + 1] (k_rot adds them up), or null
  const double* gwP0; // Gauss weight x P_0^0 / 2 per theta row
  double rotS;        // -2 / r_i
  int L;
  int fin[PROD_MAXIN];  // input field slots of four_in
};

// the two velocities of non_maxtstep (nonlinear.F90:577-603) at one point: radial
// B_r^2 / sqrt(B_r^2 E/Pm + d_r) + |u_r| and horizontal
// (B_th^2 + B_ph^2) / sqrt((B_th^2 + B_ph^2) E/Pm + d_h) + |u_h|
__device__ __forceinline__ void cfl_point(const double* v, double EPm, double E, double Pm, double dr2,
                                          double dh2, double& mr, double& mh) {
  const double vr = v[0], vt = v[1], vp = v[2], br = v[6], bt = v[7], bp = v[8];
  const double p = br * br;
  mr = fmax(mr, p / sqrt(p * EPm + dr2) + fabs(vr));
  const double q = bt * bt + bp * bp;
  mh = fmax(mh, q / sqrt(q * E / Pm + dh2) + sqrt(vt * vt + vp * vp));
}

// per-shell constants of the anelastic sets
struct ShellC { double xi0, xi1, rm1, rinv, rrr, rho, T0, dT0, eta, Cmag; };

template <int PS>
__device__ __forceinline__ void prod_point(const double* v, double* o, const ProdConst& pc, const ShellC& sh,
                                           double sn, double cs) {
  if constexpr (PS == PS_BOUSS || PS == PS_BOUSS_COMP || PS == PS_ANEL_MOM) {
    const double vr = v[0], vt = v[1], vp = v[2];
    const double wr = v[3], wt = v[4], wp = v[5];
    const double br = v[6], bt = v[7], bp = v[8];
    const double jr = v[9], jt = v[10], jp = v[11];
    double a = vt * wp - vp * wt;
    double b = vp * wr - vr * wp;
    double c = vr * wt - vt * wr;
    double Cmag = pc.Cmag;
    if constexpr (PS == PS_ANEL_MOM) {  // compressible viscous force (nonlinear.F90:93-110)
      double f = -(2.0 * sh.xi0 * sh.rm1) - sh.xi1;
      f = f - (sh.xi0 * sh.xi0) / 3.0;
      a = a + pc.Pm * vr * f;
      double d1 = 2.0 * sh.xi0 * sh.rm1 + sh.xi1;
      d1 = d1 + sh.xi0 * sh.xi0;
      b = b - pc.Pm * (sh.xi0 * wp + d1 * vt);
      c = c + pc.Pm * (sh.xi0 * wt - d1 * vp);
      Cmag = sh.Cmag;
    }
    a = a + pc.d_Cor * sn * vp;
    b = b + pc.d_Cor * cs * vp;
    c = c - pc.d_Cor * (cs * vt + sn * vr);
    a = a + Cmag * (jt * bp - jp * bt);
    b = b + Cmag * (jp * br - jr * bp);
    c = c + Cmag * (jr * bt - jt * br);
    o[0] = a; o[1] = b; o[2] = c;
    o[3] = vt * bp - vp * bt;
    o[4] = vp * br - vr * bp;
    o[5] = vr * bt - vt * br;
    if constexpr (PS != PS_ANEL_MOM) {
      const double cr = v[12], ct = v[13], cp = v[14];
      o[6] = -pc.d_qm1 * vr * cr - pc.d_qm1 * vt * ct - pc.d_qm1 * vp * cp;
    }
    if constexpr (PS == PS_BOUSS_COMP) {  // non_composition (nonlinear.F90:294-341)
      const double xr = v[15], xt = v[16], xp = v[17];
      o[7] = -pc.d_qm1c * vr * xr - pc.d_qm1c * vt * xt - pc.d_qm1c * vp * xp;
    }
  } else {  // PS_ANEL_SCAL(_COMP): inputs u 0-2, w 3-5, J 6-8, grad C 9-11, du 12-14, grad Comp 15-17
    constexpr int NI = PSet<PS>::in;
    const double vr = v[0], vt = v[1], vp = v[2];
    const double wr = v[3], wt = v[4], wp = v[5];
    const double jr = v[6], jt = v[7], jp = v[8];
    const double gr = v[9], gt = v[10], gq = v[11];
    const double dur = v[12], dutr = v[13], dupr = v[14];
    const double qv1 = v[NI], qv2 = v[NI + 1];
    double x = 2.0 * (dur * dur);
    double y = (sh.xi0 + 1.0 / sh.rrr) * vr + dur + qv1;
    x = x + 2.0 * (y * y);
    y = sh.xi0 * vr;
    x = x - 2.0 * (y * y) / 3.0;
    y = qv1 + vr / sh.rrr;
    x = x + 2.0 * (y * y);
    y = 2.0 * dutr - wp;
    x = x + y * y;
    y = 2.0 * dupr + wt;
    x = x + y * y;
    y = 2.0 * qv2 + wr;
    x = x + y * y;
    x = x + sh.eta * ((jr * jr + jp * jp + jt * jt) / (sh.rho * pc.E));
    double e = -(pc.d_qm1 * vr * gr) + (sh.dT0 / sh.T0) * gr;
    e = e - pc.d_qm1 * vt * gt;
    e = e - pc.d_qm1 * vp * gq;
    o[0] = e + (pc.Diss / sh.T0) * x;
    if constexpr (PS == PS_ANEL_SCAL_COMP) {
      const double xr = v[15], xt = v[16], xp = v[17];
      o[1] = -pc.d_qm1c * vr * xr - pc.d_qm1c * vt * xt - pc.d_qm1c * vp * xp;
    }
  }
}

// grid (2 HB, N): one half-row h = blockIdx.x (its southern and northern theta row) per
// CTA, 256 threads, up to two CTAs per SM so that one's memory waits overlap the other's
// work.  The inputs are gathered bin by bin (bin -> m-counter map, L1-cached) straight into
// the packed half spectra of the padded rows [NF][2][E (G+1)] (NF = inputs + derived rows),
// so the load phase has no barrier; barriers separate only the FFT passes and products.
constexpr int PROD_THREADS = 256;

template <int E, int G, int PS>
__global__ void __launch_bounds__(PROD_THREADS, 2) k_products(FFTPlanDev pl, int N, ProdConst pc,
                                                              const cplx* four_in, cplx* four_out) {
  constexpr int RS = E * (G + 1), P2 = E * G;
  constexpr int NF_IN = PSet<PS>::in, NDER = PSet<PS>::deriv, NF = NF_IN + NDER, NF_OUT = PSet<PS>::out;
  extern __shared__ __align__(16) unsigned char psm[];
  const int n = blockIdx.y, h = blockIdx.x, hb = h >> 1, jj = h & 1;
  const int NM = pl.NM, M = pl.M, Th = pl.Th, Th2 = pl.Th2;
  if (h >= Th2) return;  // padding half-row of an odd Th2
  double2* rows = (double2*)psm;                 // [NF][2][RS]
  const FFTTabs tabs = fft_tabs_init<E, G>((unsigned char*)(rows + (size_t)NF * 2 * RS), pl);
  const int BLK = NM * 4;                        // one field's (n, h/2) block
  const size_t fstride = (size_t)N * pl.HB * BLK;
  const size_t boff = ((size_t)n * pl.HB + hb) * BLK + jj;  // element (c, p) at boff + 2 (2c + p)
  const int tid = threadIdx.x;
  ShellC sh{};
  if constexpr (PS >= PS_ANEL_MOM) {
    const double* ref = pc.ref;
    sh.xi0 = ref[REF_XI * N + n]; sh.xi1 = ref[REF_DXI * N + n];
    sh.rho = ref[REF_RHO * N + n]; sh.T0 = ref[REF_T * N + n]; sh.dT0 = ref[REF_DT * N + n];
    sh.eta = ref[REF_ETA * N + n];
    sh.rm1 = pc.r[(size_t)2 * N + n]; sh.rinv = sh.rm1; sh.rrr = pc.r[(size_t)4 * N + n];
    sh.Cmag = pc.Pm / (pc.E * sh.rho);
  }
  // ---- gather + pack, no barrier: item (f, k), k = 0 .. P2/2, loads the (E, O) pairs of
  // bins k and P2-k (counters bin2c[.]) once, straight from this half-row's block, forms the
  // southern (E + O) and northern (E - O) half spectra and writes the packed rows at
  // positions k and P2-k (k = 0: position 0, whose partner is the Nyquist bin P2 >= M;
  // k = P2/2: its own partner).  Bins >= M are zero (dealiasing).  Batches of U items per
  // thread keep their loads in flight.
  constexpr int KH = P2 / 2 + 1, U = 3, NITEM = NF_IN * KH;
  auto put = [&](int row, int k, double2 yk, double2 ym) {
    rows[(size_t)row * RS + ppos<G>(k)] = c2r_pack(k, yk, ym, tabs.twh);
    if (k != 0 && 2 * k != P2) rows[(size_t)row * RS + ppos<G>(P2 - k)] = c2r_pack(P2 - k, ym, yk, tabs.twh);
  };
  for (int it0 = tid; it0 < NITEM; it0 += U * PROD_THREADS) {
    double2 e0[U], o0[U], e1[U], o1[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int it = it0 + u * PROD_THREADS;
      e0[u] = o0[u] = e1[u] = o1[u] = make_double2(0.0, 0.0);
      if (it < NITEM) {
        const int f = it / KH, k = it - f * KH, km = k == 0 ? P2 : P2 - k;
        const cplx* src = four_in + (size_t)pc.fin[f] * fstride + boff;
        if (k < M) {
          const int c = tabs.b2c[k];
          e0[u] = src[4 * c]; o0[u] = src[4 * c + 2];
        }
        if (km < M) {
          const int c = tabs.b2c[km];
          e1[u] = src[4 * c]; o1[u] = src[4 * c + 2];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int it = it0 + u * PROD_THREADS;
      if (it < NITEM) {
        const int f = it / KH, k = it - f * KH;
        put(f * 2, k, add2(e0[u], o0[u]), add2(e1[u], o1[u]));
        put(f * 2 + 1, k, sub2(e0[u], o0[u]), sub2(e1[u], o1[u]));
      }
    }
  }
  if constexpr (NDER > 0) {  // the qv1, qv2 rows from the u_th (input 1), u_ph (input 2) bins
    const cplx* sth = four_in + (size_t)pc.fin[1] * fstride + boff;
    const cplx* sph = four_in + (size_t)pc.fin[2] * fstride + boff;
    for (int k = tid; k < KH; k += PROD_THREADS) {  // bins k and P2-k, both sides
      const int km = k == 0 ? P2 : P2 - k;
      double2 te[2], to[2], pe[2], po[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int b = q ? km : k;
        te[q] = to[q] = pe[q] = po[q] = make_double2(0.0, 0.0);
        if (b < M) {
          const int c = tabs.b2c[b];
          te[q] = sth[4 * c]; to[q] = sth[4 * c + 2]; pe[q] = sph[4 * c]; po[q] = sph[4 * c + 2];
        }
      }
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const int j = row_theta(h, side, Th);
        const double s1 = pc.sn1[j], cot = pc.gp[j] * s1;
        double2 q1[2], q2[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const double2 t = side ? sub2(te[q], to[q]) : add2(te[q], to[q]);
          const double2 p = side ? sub2(pe[q], po[q]) : add2(pe[q], po[q]);
          const double mk = (double)((q ? km : k) * pl.Mp) * s1;
          q1[q] = make_double2(sh.rinv * (cot * t.x - mk * p.y), sh.rinv * (cot * t.y + mk * p.x));
          q2[q] = make_double2(sh.rinv * (-mk * t.y - cot * p.x), sh.rinv * (mk * t.x - cot * p.y));
        }
        put(NF_IN * 2 + side, k, q1[0], q1[1]);
        put((NF_IN + 1) * 2 + side, k, q2[0], q2[1]);
      }
    }
  }
  __syncthreads();
  // ---- inverse FFTs of the 2 NF rows
  col_pass<E, G, +1>(rows, NF * 2, tabs);
  __syncthreads();
  row_pass<E, G, +1>(rows, NF * 2, tabs);
  __syncthreads();
  // ---- products at every point (row side, sample position, part re/im), in place into 0..NF_OUT-1
  const double scale = 1.0 / (double)pl.Ph;
  constexpr bool HAS_UB = (PS == PS_BOUSS || PS == PS_BOUSS_COMP || PS == PS_ANEL_MOM);
  double cmr = 0.0, cmh = 0.0, cdr2 = 0.0, cdh2 = 0.0, EPm = 0.0;
  if (HAS_UB && pc.cflmax) {  // non_maxtstep's d per shell (nonlinear.F90:574-592)
    const double* r1 = pc.r + (size_t)4 * N;
    const double dr = n == 0 ? r1[1] - r1[0] : n == N - 1 ? r1[N - 1] - r1[N - 2]
                                              : fmin(r1[n] - r1[n - 1], r1[n + 1] - r1[n]);
    double d = (pc.E + pc.E / pc.Pm) / (2.0 * dr);
    cdr2 = d * d;
    const double drh = r1[n] / sqrt((double)(pc.L * (pc.L - 1)));
    d = pc.E / (2.0 * drh);
    cdh2 = d * d;
    EPm = pc.E / pc.Pm;
  }
  // non_rotation (nonlinear.F90:479-538) on the inner shell: sums of gwP0 (S u_ph - curl_th u)
  // sin and gwP0 B_r B_ph sin over this CTA's two theta rows (the equator row of an odd Th
  // once)
  double tv = 0.0, tm = 0.0;
  const bool torque = (PS == PS_BOUSS || PS == PS_BOUSS_COMP) && pc.rotsum && n == 0;
  for (int i = tid; i < 2 * P2; i += PROD_THREADS) {
    const int r = i / P2, pos = ppos<G>(i - r * P2);
    const int j = row_theta(h, r, Th);
    const double sn = pc.sn[j], cs = pc.gp[j];
    const bool tq = torque && !(r == 1 && (Th & 1) && h == Th2 - 1);
    double2 v[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) v[f] = rows[(size_t)(f * 2 + r) * RS + pos];
    double2 out[NF_OUT];
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      double x[NF], o[NF_OUT];
#pragma unroll
      for (int f = 0; f < NF; ++f) x[f] = part == 0 ? v[f].x : v[f].y;
      if constexpr (HAS_UB)
        if (pc.cflmax) cfl_point(x, EPm, pc.E, pc.Pm, cdr2, cdh2, cmr, cmh);
      if (tq) {
        const double gw = pc.gwP0[j];
        tv = tv + gw * ((pc.rotS * x[2] - x[4]) * sn);
        tm = tm + gw * ((x[6] * x[8]) * sn);
      }
      prod_point<PS>(x, o, pc, sh, sn, cs);
#pragma unroll
      for (int q = 0; q < NF_OUT; ++q) {
        if (part == 0) out[q].x = o[q] * scale; else out[q].y = o[q] * scale;
      }
    }
#pragma unroll
    for (int q = 0; q < NF_OUT; ++q) rows[(size_t)(q * 2 + r) * RS + pos] = out[q];
  }
  if (torque) {  // this CTA's two sums, in a fixed order, into its slots of rotsum
    __shared__ double tq[2][PROD_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
      tv += __shfl_down_sync(0xffffffffu, tv, o);
      tm += __shfl_down_sync(0xffffffffu, tm, o);
    }
    if ((tid & 31) == 0) { tq[0][tid >> 5] = tv; tq[1][tid >> 5] = tm; }
    __syncthreads();
    if (tid < 2) {
      double t = 0.0;
      for (int w = 0; w < PROD_THREADS / 32; ++w) t = t + tq[tid][w];
      pc.rotsum[2 * h + tid] = t;
    }
  }
  if constexpr (HAS_UB) {
    if (pc.cflmax) {  // CTA maxima -> the shell's slots (doubles >= 0 order as their bits)
      for (int o = 16; o > 0; o >>= 1) {
        cmr = fmax(cmr, __shfl_down_sync(0xffffffffu, cmr, o));
        cmh = fmax(cmh, __shfl_down_sync(0xffffffffu, cmh, o));
      }
      if ((tid & 31) == 0) {
        atomicMax(pc.cflmax + 2 * n, (unsigned long long)__double_as_longlong(cmr));
        atomicMax(pc.cflmax + 2 * n + 1, (unsigned long long)__double_as_longlong(cmh));
      }
    }
  }
  __syncthreads();
  // ---- forward FFTs of the product rows (spectrum back in natural order)
  row_pass<E, G, -1>(rows, NF_OUT * 2, tabs);
  __syncthreads();
  col_pass<E, G, -1>(rows, NF_OUT * 2, tabs);
  __syncthreads();
  // ---- unpack bins, fold south/north into E/O, store: a thread per (output, counter)
  // unpacks both rows once and writes the (E, O) pair, neighbours in four_off_a, with one
  // 32-byte store (the field bases are 32-byte aligned)
  const bool equator = (Th & 1) && h == Th2 - 1;  // odd Th: the equator row is counted once
  for (int i = tid; i < NF_OUT * NM; i += PROD_THREADS) {
    const int q = i / NM, c = i - q * NM;
    const int b = tabs.thm[c];
    const double2 xs = row_unpack<G>(rows + (size_t)(q * 2) * RS, b, P2, tabs.twh);
    const double2 xn = row_unpack<G>(rows + (size_t)(q * 2 + 1) * RS, b, P2, tabs.twh);
    double2 ev = add2(xs, xn);
    if (equator) { ev.x *= 0.5; ev.y *= 0.5; }
    st_global_2c(four_out + (size_t)q * fstride + four_off_a(n, c, 0, h, N, Th2), ev, sub2(xs, xn));
  }
}

// ---- standalone c2r: theta-Fourier -> phys [f][n][Ph][Th] -------------------------------
// grid (HB, N, nfields), 128 threads: the four theta rows of a half-row pair.
template <int E, int G>
__global__ void __launch_bounds__(128) k_c2r(FFTPlanDev pl, int N, const cplx* four, double* phys) {
  constexpr int RS = E * (G + 1), P2 = E * G;
  extern __shared__ __align__(16) unsigned char csm[];
  const int hb = blockIdx.x, n = blockIdx.y, f = blockIdx.z;
  const int Th = pl.Th, Th2 = pl.Th2, M = pl.M, NM = pl.NM;
  double2* rows = (double2*)csm;    // [4][RS]
  double2* sp = rows + 4 * RS;      // [4][M]
  const FFTTabs tabs = fft_tabs_init<E, G>((unsigned char*)(sp + 4 * M), pl);
  const cplx* blk = four + (((size_t)f * N + n) * pl.HB + hb) * NM * 4;
  for (int i = threadIdx.x; i < NM * 4; i += blockDim.x) stage_elem(sp, blk, tabs, M, i);
  __syncthreads();
  for (int i = threadIdx.x; i < 4 * P2; i += blockDim.x) {
    const int r = i / P2, k = i - r * P2;
    rows[r * RS + ppos<G>(k)] = c2r_pack(k, row_bin(sp, k, r >> 1, r & 1, M), row_bin(sp, k == 0 ? P2 : P2 - k, r >> 1, r & 1, M), tabs.twh);
  }
  __syncthreads();
  col_pass<E, G, +1>(rows, 4, tabs);
  __syncthreads();
  row_pass<E, G, +1>(rows, 4, tabs);
  __syncthreads();
  double* dst = phys + ((size_t)f * N + n) * (size_t)pl.Ph * Th;
  for (int i = threadIdx.x; i < 4 * P2; i += blockDim.x) {
    const int r = i / P2, pos = i - r * P2;       // pos = (G+1) t1 + t2 without the pads
    const int t1 = pos / G, t2 = pos - t1 * G, t = t1 + E * t2;
    const int h = 2 * hb + (r >> 1), side = r & 1;
    if (h >= Th2) continue;
    const int j = row_theta(h, side, Th);
    if (side && j == h) continue;  // odd Th: the equator row is written once
    const double2 z = rows[r * RS + t1 * (G + 1) + t2];
    dst[(size_t)(2 * t) * Th + j] = z.x;
    dst[(size_t)(2 * t + 1) * Th + j] = z.y;
  }
}

// ---- standalone r2c: phys [f][n][Ph][Th] -> folded theta-Fourier, analysis layout ---------
template <int E, int G>
__global__ void __launch_bounds__(128) k_r2c(FFTPlanDev pl, int N, const double* phys, cplx* four) {
  constexpr int RS = E * (G + 1), P2 = E * G;
  extern __shared__ __align__(16) unsigned char rsm[];
  const int hb = blockIdx.x, n = blockIdx.y, f = blockIdx.z;
  const int Th = pl.Th, Th2 = pl.Th2, NM = pl.NM;
  double2* rows = (double2*)rsm;  // [4][RS]
  const FFTTabs tabs = fft_tabs_init<E, G>((unsigned char*)(rows + 4 * RS), pl);
  const double scale = 1.0 / (double)pl.Ph;
  const double* src = phys + ((size_t)f * N + n) * (size_t)pl.Ph * Th;
  for (int i = threadIdx.x; i < 4 * P2; i += blockDim.x) {
    const int r = i / P2, pos = i - r * P2;
    const int t1 = pos / G, t2 = pos - t1 * G, t = t1 + E * t2;
    const int h = 2 * hb + (r >> 1);
    const int j = row_theta(h < Th2 ? h : 2 * hb, r & 1, Th);
    rows[r * RS + t1 * (G + 1) + t2] =
        make_double2(src[(size_t)(2 * t) * Th + j] * scale, src[(size_t)(2 * t + 1) * Th + j] * scale);
  }
  __syncthreads();
  row_pass<E, G, -1>(rows, 4, tabs);
  __syncthreads();
  col_pass<E, G, -1>(rows, 4, tabs);
  __syncthreads();
  cplx* fld = four + (size_t)f * N * pl.HB * NM * 4;  // analysis layout (four_off_a)
  for (int i = threadIdx.x; i < NM * 2; i += blockDim.x) {
    const int c = i >> 1, q = i & 1, hh = 2 * hb + q, b = tabs.thm[c];
    if (hh >= Th2) continue;
    const double2 xs = row_unpack<G>(rows + (2 * q) * RS, b, P2, tabs.twh);
    const double2 xn = row_unpack<G>(rows + (2 * q + 1) * RS, b, P2, tabs.twh);
    double2 ev = add2(xs, xn);
    if ((Th & 1) && hh == Th2 - 1) { ev.x *= 0.5; ev.y *= 0.5; }
    fld[four_off_a(n, c, 0, hh, N, Th2)] = ev;
    fld[four_off_a(n, c, 1, hh, N, Th2)] = sub2(xs, xn);
  }
}

// qv1, qv2 of tra_qst2rtp_vel (transform.fftw3.F90:678-700) from the u_th, u_ph
// theta-Fourier rows, on the even/odd half-grid sums: cot theta is odd about the equator,
// so it swaps E and O, while 1/sin theta keeps them (the identity is stated at PS_ANEL_SCAL).
__global__ void k_qv_four(FFTPlanDev pl, int N, const double* rinv, const double* gp, const double* sn1,
                          const cplx* th, const cplx* ph, cplx* q1, cplx* q2) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // (n, hb, c, h & 1)
  const size_t total = (size_t)N * pl.HB * pl.NM * 2;
  if (i >= total) return;
  const int hh = (int)(i & 1), c = (int)((i >> 1) % pl.NM);
  const size_t nb = (i >> 1) / pl.NM;
  const int hb = (int)(nb % pl.HB), n = (int)(nb / pl.HB), h = 2 * hb + hh;
  const size_t oE = four_off(n, c, 0, h, pl.NM, pl.HB), oO = four_off(n, c, 1, h, pl.NM, pl.HB);
  if (h >= pl.Th2) {
    q1[oE] = q1[oO] = q2[oE] = q2[oO] = make_double2(0.0, 0.0);
    return;
  }
  const double s1 = sn1[h], cot = gp[h] * s1, ri = rinv[n];
  const double mk = (double)(pl.thm[c] * pl.Mp) * s1;
  const double2 te = th[oE], to = th[oO], pe = ph[oE], po = ph[oO];
  // i mk (x + i y) = (-mk y, mk x)
  q1[oE] = make_double2(ri * (cot * to.x - mk * pe.y), ri * (cot * to.y + mk * pe.x));
  q1[oO] = make_double2(ri * (cot * te.x - mk * po.y), ri * (cot * te.y + mk * po.x));
  q2[oE] = make_double2(ri * (-mk * te.y - cot * po.x), ri * (mk * te.x - cot * po.y));
  q2[oO] = make_double2(ri * (-mk * to.y - cot * pe.x), ri * (mk * to.x - cot * pe.y));
}

FFTPlanDev make_plan(lsd_ctx* ctx) {
  FFTPlanDev pl;
  pl.P2 = ctx->P2; pl.Ph = ctx->Ph; pl.M = ctx->M; pl.NM = ctx->NM; pl.Th = ctx->Th; pl.Th2 = ctx->Th2;
  pl.HB = ctx->HB; pl.Mp = ctx->Mp;
  pl.tw2 = ctx->d_tw2; pl.twh = ctx->d_twh; pl.thm = ctx->d_thm; pl.bin2c = ctx->d_bin2c;
  return pl;
}

// (E, G) pairs: P2 = 3 * 2^a or 9 * 2^a with the power of two split off up to 16 (the
// default plan), and with one factor 2 moved to the column DFT (G = 8, the autotuner's
// alternative for P2 = 48 .. 288)
template <class F>
int dispatch_EG(int E, int G, F&& f) {
#define LSD_EG(e, g) if (E == e && G == g) return f(std::integral_constant<int, e>(), std::integral_constant<int, g>());
  LSD_EG(3, 1) LSD_EG(3, 2) LSD_EG(3, 4) LSD_EG(3, 8) LSD_EG(3, 16)
  LSD_EG(9, 1) LSD_EG(9, 2) LSD_EG(9, 4) LSD_EG(9, 8) LSD_EG(9, 16)
  LSD_EG(6, 16) LSD_EG(12, 16) LSD_EG(18, 16) LSD_EG(24, 16)
  LSD_EG(6, 8) LSD_EG(12, 8) LSD_EG(18, 8) LSD_EG(24, 8) LSD_EG(36, 8)
#undef LSD_EG
  return -1;
}

}  // namespace

bool lsd_fft_compiled(int E, int G) { return dispatch_EG(E, G, [](auto, auto) { return 0; }) == 0; }

// shared memory of the products kernel with the plan (E, G) for nfields staged rows
size_t lsd_products_smem_for(int nfields, int P2, int E, int G, int NM) {
  return sizeof(double2) * ((size_t)nfields * 2 * E * (G + 1)) + fft_tab_bytes(P2, E, G, NM);
}
size_t lsd_products_smem_eg(const lsd_ctx* ctx, int E, int G) {
  const bool comp = ctx->cfg.comp_tstep != 0;
  int nf = comp ? 18 : 15;
  if (!ctx->cfg.boussinesq) nf = (comp ? 18 : 15) + 2;
  return lsd_products_smem_for(nf, ctx->P2, E, G, ctx->NM);
}

// P2 = E G with G the power-of-two part of P2 capped at 16; (E, G) must be instantiated.
bool lsd_fft_plan(lsd_ctx* c) {
  int G = 1;
  while (G < 16 && c->P2 % (2 * G) == 0) G *= 2;
  const int E = c->P2 / G;
  c->fftG = G;
  c->fftE = E;
  return dispatch_EG(E, G, [](auto, auto) { return 0; }) == 0;
}

int lsd_launch_c2r(lsd_ctx* ctx, const cplx* four, double* phys, int nfields) {
  FFTPlanDev pl = make_plan(ctx);
  dim3 grid(ctx->HB, ctx->N, nfields);
  const size_t smem = sizeof(double2) * 4 * (ctx->fftE * (ctx->fftG + 1) + ctx->M) +
                      fft_tab_bytes(ctx->P2, ctx->fftE, ctx->fftG, ctx->NM);
  int rc = dispatch_EG(ctx->fftE, ctx->fftG, [&](auto e, auto g) {
    constexpr int E = decltype(e)::value, G = decltype(g)::value;
    cudaFuncSetAttribute(k_c2r<E, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_c2r<E, G><<<grid, 128, smem, ctx->stream>>>(pl, ctx->N, four, phys);
    return 0;
  });
  if (rc) return lsd_fail(ctx, LSD_EARG, "FFT length not supported");
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_c2r: ") + cudaGetErrorString(e));
  return LSD_OK;
}

int lsd_launch_r2c(lsd_ctx* ctx, const double* phys, cplx* four, int nfields) {
  FFTPlanDev pl = make_plan(ctx);
  dim3 grid(ctx->HB, ctx->N, nfields);
  const size_t smem = sizeof(double2) * 4 * ctx->fftE * (ctx->fftG + 1) +
                      fft_tab_bytes(ctx->P2, ctx->fftE, ctx->fftG, ctx->NM);
  int rc = dispatch_EG(ctx->fftE, ctx->fftG, [&](auto e, auto g) {
    constexpr int E = decltype(e)::value, G = decltype(g)::value;
    cudaFuncSetAttribute(k_r2c<E, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_r2c<E, G><<<grid, 128, smem, ctx->stream>>>(pl, ctx->N, phys, four);
    return 0;
  });
  if (rc) return lsd_fail(ctx, LSD_EARG, "FFT length not supported");
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_r2c: ") + cudaGetErrorString(e));
  return LSD_OK;
}

namespace {
template <int PS>
int launch_products_set(lsd_ctx* ctx, const ProdConst& pc, const cplx* four_in, cplx* four_out) {
  FFTPlanDev pl = make_plan(ctx);
  constexpr int NF = PSet<PS>::in + PSet<PS>::deriv;
  const size_t smem = sizeof(double2) * ((size_t)NF * 2 * ctx->fftE * (ctx->fftG + 1)) +
                      fft_tab_bytes(ctx->P2, ctx->fftE, ctx->fftG, ctx->NM);
  if (smem > 224 * 1024) return lsd_fail(ctx, LSD_EARG, "products: FFT rows do not fit in shared memory");
  dim3 grid(2 * ctx->HB, ctx->N);
  int rc = dispatch_EG(ctx->fftE, ctx->fftG, [&](auto e, auto g) {
    constexpr int E = decltype(e)::value, G = decltype(g)::value;
    cudaFuncSetAttribute(k_products<E, G, PS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_products<E, G, PS><<<grid, PROD_THREADS, smem, ctx->stream>>>(pl, ctx->N, pc, four_in, four_out);
    return 0;
  });
  if (rc) return lsd_fail(ctx, LSD_EARG, "FFT length not supported");
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_products: ") + cudaGetErrorString(e));
  return LSD_OK;
}
}  // namespace

// tim_cfl_dt from the per-shell maxima (nonlinear.F90:593-605); one thread, shells in order
__global__ void k_cfl_finish(int N, int L, double E, double Pm, const double* r, const unsigned long long* cflmax,
                             double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double* r1 = r + (size_t)4 * N;
  double cfl = 1e99;
  for (int n = 0; n < N; ++n) {
    const double dr = n == 0 ? r1[1] - r1[0] : n == N - 1 ? r1[N - 1] - r1[N - 2]
                                              : fmin(r1[n] - r1[n - 1], r1[n + 1] - r1[n]);
    const double mr = __longlong_as_double((long long)cflmax[2 * n]);
    if (mr != 0.0) cfl = fmin(cfl, dr / mr);
    const double drh = r1[n] / sqrt((double)(L * (L - 1)));
    const double mh = __longlong_as_double((long long)cflmax[2 * n + 1]);
    if (mh != 0.0) cfl = fmin(cfl, drh / mh);
  }
  cfl = fmin(cfl, E / Pm);
  cfl = fmin(cfl, sqrt(E));
  *out = cfl;
}

int lsd_launch_cfl_finish(lsd_ctx* ctx) {
  k_cfl_finish<<<1, 32, 0, ctx->stream>>>(ctx->N, ctx->L, ctx->cfg.E, ctx->cfg.Pm, ctx->d_r,
                                          (const unsigned long long*)ctx->d_cfl, ctx->d_cfl + 2 * ctx->N);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_cfl_finish: ") + cudaGetErrorString(e));
  return LSD_OK;
}

int lsd_launch_qv(lsd_ctx* ctx, const cplx* th, const cplx* ph, cplx* qv1, cplx* qv2) {
  FFTPlanDev pl = make_plan(ctx);
  const size_t total = (size_t)ctx->N * ctx->HB * ctx->NM * 2;
  k_qv_four<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(pl, ctx->N, ctx->d_r + (size_t)2 * ctx->N,
                                                                      ctx->d_gp, ctx->d_sn1, th, ph, qv1, qv2);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_qv_four: ") + cudaGetErrorString(e));
  return LSD_OK;
}

size_t lsd_products_smem(const lsd_ctx* ctx) { return lsd_products_smem_eg(ctx, ctx->fftE, ctx->fftG); }

// four_in: the synthesised fields in the FFT layout, slots u 0-2, curl u 3-5, B 6-8,
// curl B 9-11, grad C 12-14, grad Comp 15-17 (composition), then (anelastic) dr u_r,
// dr u_th, dr u_ph; four_out: the products in the analysis layout, slots 0-2 momentum,
// 3-5 u x B, 6 codensity, 7 composition.
int lsd_launch_products(lsd_ctx* ctx, const cplx* four_in, cplx* four_out) {
  ProdConst pc;
  const lsd_config& c = ctx->cfg;
  pc.d_Cor = 2.0 * c.Pm / c.E;
  pc.Cmag = 2 * c.Pm / c.E;
  pc.d_qm1 = c.Pr / c.Pm;
  pc.d_qm1c = c.Sc / c.Pm;
  pc.Pm = c.Pm;
  pc.E = c.E;
  pc.Diss = pc.d_qm1 * pc.d_qm1 / c.Ra;
  pc.sn = ctx->d_sn;
  pc.gp = ctx->d_gp;
  pc.sn1 = ctx->d_sn1;
  pc.r = ctx->d_r;
  pc.ref = ctx->d_ref;
  pc.L = ctx->L;
  pc.cflmax = c.timestep < 0 ? (unsigned long long*)ctx->d_cfl : nullptr;
  pc.rotsum = c.rot_tstep ? ctx->d_rot + ROT_NSLOT : nullptr;
  pc.gwP0 = ctx->d_gwP0;
  pc.rotS = -2.0 / (c.rratio / (1.0 - c.rratio));  // r(1,1) = r_i
  const bool comp = c.comp_tstep != 0;
  const size_t FF = (size_t)ctx->N * ctx->HB * ctx->NM * 4;
  if (c.boussinesq) {
    for (int f = 0; f < PROD_MAXIN; ++f) pc.fin[f] = f;
    return comp ? launch_products_set<PS_BOUSS_COMP>(ctx, pc, four_in, four_out)
                : launch_products_set<PS_BOUSS>(ctx, pc, four_in, four_out);
  }
  for (int f = 0; f < PROD_MAXIN; ++f) pc.fin[f] = f < 12 ? f : 0;
  int rc = launch_products_set<PS_ANEL_MOM>(ctx, pc, four_in, four_out);
  if (rc) return rc;
  const int du = comp ? 18 : 15;
  const int sl[PROD_MAXIN] = {0, 1, 2, 3, 4, 5, 9, 10, 11, 12, 13, 14, du, du + 1, du + 2, 15, 16, 17};
  for (int f = 0; f < PROD_MAXIN; ++f) pc.fin[f] = sl[f];
  return comp ? launch_products_set<PS_ANEL_SCAL_COMP>(ctx, pc, four_in, four_out + 6 * FF)
              : launch_products_set<PS_ANEL_SCAL>(ctx, pc, four_in, four_out + 6 * FF);
}
