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
// Each complex FFT of length P2 = E G (G a power of two <= 32) runs in the registers of
// G lanes: lane l holds E values.  The inverse is a lane-parallel radix-2 DIF over the G
// lanes (shuffles), a twiddle w^(g k1) and an E-point DFT in registers; the forward
// transform is its mirror (E-point DFT, twiddle, radix-2 DIT over the lanes).  Physical
// samples come out of the inverse in a lane-permuted order and the forward transform
// takes them back in that order, so the point-wise products never need a reordering.
// Every shuffle runs with all 32 lanes of the warp: task loops advance warp by warp and
// lanes without a task compute a dummy row whose results are dropped.
//
// The theta-Fourier rows are stored in half-row pairs ([n][h/2][m-counter][E/O][h%2],
// four_off); one CTA of the fused kernel owns one pair (four full theta rows: the
// southern and northern row of each half-row), reads the 15 synthesised fields of u,
// curl u, B, curl B and grad C as contiguous 8 KB blocks, transforms them, forms
//   u x (curl u) + Coriolis + Lorentz      (nonlinear.F90:70-146, Boussinesq)
//   -(Pr/Pm) u . grad C                     (nonlinear.F90:269-272)
//   u x B                                   (nonlinear.F90:421-430)
// at every grid point in shared memory, transforms the 7 results back and writes their
// folded theta-Fourier rows.  Physical-space fields never touch HBM.
#include <algorithm>
#include <type_traits>

#include "lsd_common.cuh"

namespace {

constexpr unsigned FULL = 0xffffffffu;

struct FFTPlanDev {
  int P2, Ph, M, NM, Th, Th2, HB, G, lgG;
  const double2* tw2;  // e^{+2 pi i k/P2}, k < P2
  const double2* twh;  // e^{+2 pi i k/Ph}, k < Ph
  const int* thm;      // m-counter -> bin
  const int* bin2c;    // bin b < M -> m-counter
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
__device__ __forceinline__ double2 shfl_xor2(double2 v, int m) {
  return make_double2(__shfl_xor_sync(FULL, v.x, m), __shfl_xor_sync(FULL, v.y, m));
}
__device__ __forceinline__ double2 shfl2(double2 v, int src) {
  return make_double2(__shfl_sync(FULL, v.x, src), __shfl_sync(FULL, v.y, src));
}
__device__ __forceinline__ int brev_bits(int l, int bits) {
  return bits ? (int)(__brev((unsigned)l) >> (32 - bits)) : 0;
}

// In-register DFT of length N (mixed radix 2/3, decimation in time) with the twiddles of
// the full length EF: w[j] = e^{+2 pi i j / EF} (a shared-memory table, read as
// broadcasts); SIGN +1 inverse, -1 forward.
template <int SIGN>
__device__ __forceinline__ double2 twid(double2 a, double2 w) { return SIGN > 0 ? cmul(a, w) : cmulc(a, w); }

template <int N, int EF, int SIGN>
__device__ __forceinline__ void rdft(double2 (&x)[N], const double2* w) {
  if constexpr (N == 1) {
    return;
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
//   wst[s][l] = e^{+2 pi i (l mod h) / (2h)}, h = 2^s    lane-stage twiddles, [s][lane]
//   wlt[t][l] = e^{+2 pi i t l / P2}                     inter-step twiddles, [t][lane]
//   twE[j]    = e^{+2 pi i j / E}                        register-DFT twiddles (broadcast)
//   thm[c]    = FFT bin of m-counter c
// Lane-indexed tables are read at consecutive addresses by consecutive lanes.
struct FFTTabs {
  double2* wst;
  double2* wlt;
  double2* twE;
  int* thm;
};

__host__ __device__ __forceinline__ size_t fft_tab_bytes(int G, int E, int NM) {
  return sizeof(double2) * ((size_t)5 * G + (size_t)E * G + E) + sizeof(int) * (size_t)((NM + 3) & ~3);
}

// carve the tables out of `base` (16-byte aligned) and fill them; ends with a barrier
template <int E>
__device__ __forceinline__ FFTTabs fft_tabs_init(unsigned char* base, const FFTPlanDev& pl) {
  const int G = pl.G;
  FFTTabs t;
  t.wst = (double2*)base;
  t.wlt = t.wst + 5 * G;
  t.twE = t.wlt + E * G;
  t.thm = (int*)(t.twE + E);
  for (int i = threadIdx.x; i < 5 * G; i += blockDim.x) {
    const int s = i / G, l = i % G, h = 1 << s;
    t.wst[i] = h < G ? __ldg(&pl.tw2[E * (l & (h - 1)) * (G / (2 * h))]) : make_double2(1.0, 0.0);
  }
  for (int i = threadIdx.x; i < E * G; i += blockDim.x) t.wlt[i] = __ldg(&pl.tw2[(i / G) * (i % G)]);
  for (int i = threadIdx.x; i < E; i += blockDim.x) t.twE[i] = __ldg(&pl.tw2[G * i]);
  for (int i = threadIdx.x; i < pl.NM; i += blockDim.x) t.thm[i] = __ldg(&pl.thm[i]);
  __syncthreads();
  return t;
}

// Inverse (e^{+i}) FFT of length P2 = E G on G lanes.
//   In:  v[k1] = Z[l + G k1]        (lane l holds every G-th bin from l)
//   Out: v[t1] = x[t1 + E brev(l)]  (brev over log2 G bits)
// x[t1 + E t2] = sum_k2 w_G^(t2 k2) w^(t1 k2) sum_k1 w_E^(t1 k1) Z[k2 + G k1].
template <int E>
__device__ __forceinline__ void wfft_inv(double2 (&v)[E], int l, const FFTPlanDev& pl, const FFTTabs& t) {
  const int G = pl.G;
  rdft<E, E, +1>(v, t.twE);
#pragma unroll
  for (int k = 1; k < E; ++k) v[k] = cmul(v[k], t.wlt[k * G + l]);
#pragma unroll
  for (int s = 4; s >= 0; --s) {  // radix-2 DIF over the lanes (natural -> bit-reversed)
    const int h = 1 << s;
    if (h >= G) continue;
    const bool up = l & h;
    const double2 w = t.wst[s * G + l];
#pragma unroll
    for (int k = 0; k < E; ++k) {
      const double2 p = shfl_xor2(v[k], h);
      v[k] = up ? cmul(sub2(p, v[k]), w) : add2(v[k], p);
    }
  }
}

// Forward (e^{-i}) FFT, the mirror of wfft_inv.
//   In:  v[t1] = x[t1 + E brev(l)]      Out: v[k1] = X[l + G k1]
template <int E>
__device__ __forceinline__ void wfft_fwd(double2 (&v)[E], int l, const FFTPlanDev& pl, const FFTTabs& t) {
  const int G = pl.G;
#pragma unroll
  for (int s = 0; s <= 4; ++s) {  // radix-2 DIT over the lanes (bit-reversed -> natural)
    const int h = 1 << s;
    if (h >= G) continue;
    const bool up = l & h;
    const double2 w = t.wst[s * G + l];
#pragma unroll
    for (int k = 0; k < E; ++k) {
      const double2 send = up ? cmulc(v[k], w) : v[k];
      const double2 recv = shfl_xor2(send, h);
      v[k] = up ? sub2(recv, send) : add2(send, recv);
    }
  }
#pragma unroll
  for (int k = 1; k < E; ++k) v[k] = cmulc(v[k], t.wlt[k * G + l]);
  rdft<E, E, -1>(v, t.twE);
}

// Half-spectrum packing for the c2r: Z[k] from Y[k] and conj(Y[P2-k]) (Y[P2] = Nyquist = 0;
// the imaginary part of the DC bin is ignored).
__device__ __forceinline__ double2 c2r_pack(int k, double2 yk, double2 ymk, const FFTPlanDev& pl) {
  const double2 yc = conj2(ymk);
  if (k == 0) yk.y = 0.0;
  const double2 s = add2(yk, yc), d = sub2(yk, yc);
  const double2 wd = cmul(__ldg(&pl.twh[k]), d);
  return make_double2(s.x - wd.y, s.y + wd.x);  // s + i w d
}
// Bin k < P2 of the real spectrum from Z[k] and Z[P2-k] (Z[0] for k = 0).
__device__ __forceinline__ double2 r2c_unpack(int k, double2 zk, double2 zmk, const FFTPlanDev& pl) {
  if (k == 0) return make_double2(zk.x + zk.y, 0.0);
  const double2 zc = conj2(zmk);
  const double2 A = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
  const double2 Bi = make_double2(0.5 * (zk.x - zc.x), 0.5 * (zk.y - zc.y));  // i B
  const double2 B = make_double2(Bi.y, -Bi.x);
  return add2(A, cmulc(B, __ldg(&pl.twh[k])));
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

// Pack + inverse FFT of one row from a staged field.
template <int E>
__device__ __forceinline__ void row_c2r(double2 (&v)[E], const double2* sp, int jj, int side, int l,
                                        const FFTPlanDev& pl, const FFTTabs& t) {
  const int P2 = pl.P2, G = pl.G;
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) {
    const int k = l + G * k1;
    v[k1] = c2r_pack(k, row_bin(sp, k, jj, side, pl.M), row_bin(sp, P2 - k, jj, side, pl.M), pl);
  }
  wfft_inv<E>(v, l, pl, t);
}

// Forward FFT of one row of physical samples (lane order) + unpack of bins k = l + G k1.
// Z[P2 - k] lives in lane G - l, register E - 1 - k1 (l > 0), or in lane 0, register E - k1.
template <int E>
__device__ __forceinline__ void row_r2c(double2 (&v)[E], int l, int lane0, const FFTPlanDev& pl, const FFTTabs& t) {
  const int G = pl.G;
  wfft_fwd<E>(v, l, pl, t);
  double2 out[E];
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) {
    const double2 za = shfl2(v[E - 1 - k1], lane0 + (G - l) % G);
    const double2 zb = shfl2(v[(E - k1) % E], lane0);
    out[k1] = r2c_unpack(l + G * k1, v[k1], l ? za : zb, pl);
  }
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) v[k1] = out[k1];
}

// ---- fused: 15 theta-Fourier inputs -> products -> 7 theta-Fourier outputs -------------
struct ProdConst {
  double d_Cor, Cmag, d_qm1;
  const double* sn;  // sin(theta_j)
  const double* gp;  // cos(theta_j)
};

constexpr int NF_IN = 15, NF_OUT = 7;

// grid (HB or 2 HB, N); RPC = 4 rows (both half-rows of the pair) or 2 (one half-row,
// blockIdx.x = h, for long rows).  Shared memory: the physical rows [NF_IN][RPC][P2]
// (double2, lane order), FPR staged fields [FPR][4][M], the FFT tables.
template <int E>
__global__ void __launch_bounds__(512) k_products(FFTPlanDev pl, int N, ProdConst pc, const cplx* four_in,
                                                  cplx* four_out, int RPC, int FPR) {
  extern __shared__ __align__(16) unsigned char psm[];
  const int n = blockIdx.y;
  const int hb = RPC == 4 ? blockIdx.x : blockIdx.x >> 1;
  const int jj0 = RPC == 4 ? 0 : (blockIdx.x & 1);
  const int P2 = pl.P2, G = pl.G, NM = pl.NM, M = pl.M, Th = pl.Th, Th2 = pl.Th2;
  const int BLK = NM * 4;  // complex values of one field's (n, h/2) block
  double2* phys = (double2*)psm;
  double2* stage = phys + (size_t)NF_IN * RPC * P2;
  const FFTTabs tabs = fft_tabs_init<E>((unsigned char*)(stage + (size_t)FPR * 4 * M), pl);
  const size_t fstride = (size_t)N * pl.HB * BLK;
  const size_t boff = ((size_t)n * pl.HB + hb) * BLK;  // the CTA's block in every field
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int sgw = 32 / G, l = lane % G, lane0 = lane - l;
  const int sg = warp * sgw + lane / G;
  // ---- inverse transforms, FPR fields per round: stage their blocks (coalesced reads),
  //      then sub-group sg takes (field f0 + sg / RPC, row sg % RPC)
  for (int f0 = 0; f0 < NF_IN; f0 += FPR) {
    const int nf = min(FPR, NF_IN - f0);
    for (int i = threadIdx.x; i < nf * BLK; i += blockDim.x) {
      const int fi = i / BLK;
      stage_elem(stage + (size_t)fi * 4 * M, four_in + (size_t)(f0 + fi) * fstride + boff, tabs, M, i - fi * BLK);
    }
    __syncthreads();
    const int fi = sg / RPC, r = sg % RPC;
    const int jj = jj0 + (r >> 1), side = r & 1;
    const bool act = fi < nf && 2 * hb + jj < Th2;
    double2 v[E];
    row_c2r<E>(v, stage + (size_t)(fi < nf ? fi : 0) * 4 * M, jj, side, l, pl, tabs);
    if (act) {
      double2* dst = phys + ((size_t)(f0 + fi) * RPC + r) * P2;
#pragma unroll
      for (int e = 0; e < E; ++e) dst[e * G + l] = v[e];
    }
    __syncthreads();
  }
  // ---- products at every point (row r, position i, part re/im), in place into slots 0..6
  const double scale = 1.0 / (double)pl.Ph;
  for (int i = threadIdx.x; i < RPC * P2; i += blockDim.x) {
    const int r = i / P2, pos = i - r * P2;
    const int h = 2 * hb + jj0 + (r >> 1);
    if (h >= Th2) continue;
    const int j = row_theta(h, r & 1, Th);
    const double sn = pc.sn[j], cs = pc.gp[j];
    double2 v[NF_IN];
#pragma unroll
    for (int f = 0; f < NF_IN; ++f) v[f] = phys[((size_t)f * RPC + r) * P2 + pos];
    double2 out[NF_OUT];
#pragma unroll
    for (int part = 0; part < 2; ++part) {
#define G_(f) (part == 0 ? v[f].x : v[f].y)
      const double vr = G_(0), vt = G_(1), vp = G_(2);
      const double wr = G_(3), wt = G_(4), wp = G_(5);
      const double br = G_(6), bt = G_(7), bp = G_(8);
      const double jr = G_(9), jt = G_(10), jp = G_(11);
      const double cr = G_(12), ct = G_(13), cp = G_(14);
#undef G_
      double a = vt * wp - vp * wt;
      double b = vp * wr - vr * wp;
      double c = vr * wt - vt * wr;
      a = a + pc.d_Cor * sn * vp;
      b = b + pc.d_Cor * cs * vp;
      c = c - pc.d_Cor * (cs * vt + sn * vr);
      a = a + pc.Cmag * (jt * bp - jp * bt);
      b = b + pc.Cmag * (jp * br - jr * bp);
      c = c + pc.Cmag * (jr * bt - jt * br);
      const double e0 = vt * bp - vp * bt;
      const double e1 = vp * br - vr * bp;
      const double e2 = vr * bt - vt * br;
      const double cod = -pc.d_qm1 * vr * cr - pc.d_qm1 * vt * ct - pc.d_qm1 * vp * cp;
      const double o[NF_OUT] = {a, b, c, e0, e1, e2, cod};
#pragma unroll
      for (int q = 0; q < NF_OUT; ++q) {
        if (part == 0) out[q].x = o[q] * scale; else out[q].y = o[q] * scale;
      }
    }
#pragma unroll
    for (int q = 0; q < NF_OUT; ++q) phys[((size_t)q * RPC + r) * P2 + pos] = out[q];
  }
  __syncthreads();
  // ---- forward transforms: task = (output, row); bins b < M back into the row's slot
  for (int t0 = warp * sgw; t0 < NF_OUT * RPC; t0 += nw * sgw) {
    const int t = t0 + lane / G;
    const int tt = t < NF_OUT * RPC ? t : t0;  // lanes without a task redo a valid one
    const int q = tt / RPC, r = tt % RPC;
    const bool act = t < NF_OUT * RPC && 2 * hb + jj0 + (r >> 1) < Th2;
    double2* slot = phys + ((size_t)q * RPC + r) * P2;
    double2 v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = slot[e * G + l];
    row_r2c<E>(v, l, lane0, pl, tabs);
    __syncwarp();
    if (act) {
#pragma unroll
      for (int k1 = 0; k1 < E; ++k1) {
        const int b = l + G * k1;
        if (b < M) slot[b] = v[k1];
      }
    }
    __syncwarp();
  }
  __syncthreads();
  // ---- fold south/north into E/O and store the output blocks (contiguous per field)
  const int njj = RPC / 2;
  for (int i = threadIdx.x; i < NF_OUT * NM * 2 * njj; i += blockDim.x) {
    const int q = i / (NM * 2 * njj), rem = i % (NM * 2 * njj);
    const int c = rem / (2 * njj), p = (rem / njj) % 2, jr = rem % njj;
    const int jj = jj0 + jr, h = 2 * hb + jj;
    if (h >= Th2) continue;
    const int b = tabs.thm[c];
    const double2 xs = phys[((size_t)q * RPC + 2 * jr) * P2 + b];
    const double2 xn = phys[((size_t)q * RPC + 2 * jr + 1) * P2 + b];
    double2 val = p == 0 ? add2(xs, xn) : sub2(xs, xn);
    if (p == 0 && (Th & 1) && h == Th2 - 1) { val.x *= 0.5; val.y *= 0.5; }  // odd Th: equator once
    four_out[q * fstride + boff + (c * 2 + p) * 2 + jj] = val;
  }
}

// ---- standalone c2r: theta-Fourier -> phys [f][n][Ph][Th] -------------------------------
// grid (HB, N, nfields), 128 threads: the four theta rows of a half-row pair, G lanes each
// (sub-groups beyond the four rows redo row 0 and drop it).
template <int E>
__global__ void __launch_bounds__(128) k_c2r(FFTPlanDev pl, int N, const cplx* four, double* phys) {
  extern __shared__ __align__(16) unsigned char csm[];
  const int hb = blockIdx.x, n = blockIdx.y, f = blockIdx.z;
  const int G = pl.G, Th = pl.Th, Th2 = pl.Th2, M = pl.M, NM = pl.NM;
  double2* sp = (double2*)csm;  // [4][M]
  const FFTTabs tabs = fft_tabs_init<E>((unsigned char*)(sp + 4 * M), pl);
  const cplx* blk = four + (((size_t)f * N + n) * pl.HB + hb) * NM * 4;
  for (int i = threadIdx.x; i < NM * 4; i += blockDim.x) stage_elem(sp, blk, tabs, M, i);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int l = lane % G;
  const int grp = warp * (32 / G) + lane / G;
  const int r = grp < 4 ? grp : 0;
  const int jj = r >> 1, side = r & 1, h = 2 * hb + jj;
  double2 v[E];
  row_c2r<E>(v, sp, jj, side, l, pl, tabs);
  const int j = row_theta(h, side, Th);
  if (grp >= 4 || h >= Th2 || (side && j == h)) return;  // odd Th: the equator row is written once
  double* dst = phys + ((size_t)f * N + n) * (size_t)pl.Ph * Th;
  const int t2 = brev_bits(l, pl.lgG);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int t = e + E * t2;
    dst[(size_t)(2 * t) * Th + j] = v[e].x;
    dst[(size_t)(2 * t + 1) * Th + j] = v[e].y;
  }
}

// ---- standalone r2c: phys [f][n][Ph][Th] -> folded theta-Fourier --------------------------
template <int E>
__global__ void __launch_bounds__(128) k_r2c(FFTPlanDev pl, int N, const double* phys, cplx* four) {
  extern __shared__ __align__(16) unsigned char rsm[];
  const int hb = blockIdx.x, n = blockIdx.y, f = blockIdx.z;
  const int G = pl.G, Th = pl.Th, Th2 = pl.Th2, M = pl.M, NM = pl.NM;
  double2* bins = (double2*)rsm;  // [4][M]
  const FFTTabs tabs = fft_tabs_init<E>((unsigned char*)(bins + 4 * M), pl);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int l = lane % G, lane0 = lane - l;
  const int grp = warp * (32 / G) + lane / G;
  const int r = grp < 4 ? grp : 0;
  const int jj = r >> 1, side = r & 1, h = 2 * hb + jj;
  const double scale = 1.0 / (double)pl.Ph;
  const int j = row_theta(h < Th2 ? h : 2 * hb, side, Th);
  const double* src = phys + ((size_t)f * N + n) * (size_t)pl.Ph * Th;
  const int t2 = brev_bits(l, pl.lgG);
  double2 v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int t = e + E * t2;
    v[e] = make_double2(src[(size_t)(2 * t) * Th + j] * scale, src[(size_t)(2 * t + 1) * Th + j] * scale);
  }
  row_r2c<E>(v, l, lane0, pl, tabs);
  if (grp < 4) {
#pragma unroll
    for (int k1 = 0; k1 < E; ++k1) {
      const int b = l + G * k1;
      if (b < M) bins[r * M + b] = v[k1];
    }
  }
  __syncthreads();
  cplx* blk = four + (((size_t)f * N + n) * pl.HB + hb) * NM * 4;
  for (int i = threadIdx.x; i < NM * 4; i += blockDim.x) {
    const int c = i >> 2, p = (i >> 1) & 1, q = i & 1, hh = 2 * hb + q, b = tabs.thm[c];
    if (hh >= Th2) continue;
    const double2 xs = bins[(2 * q) * M + b], xn = bins[(2 * q + 1) * M + b];
    double2 val = p == 0 ? add2(xs, xn) : sub2(xs, xn);
    if (p == 0 && (Th & 1) && hh == Th2 - 1) { val.x *= 0.5; val.y *= 0.5; }
    blk[i] = val;
  }
}

FFTPlanDev make_plan(lsd_ctx* ctx) {
  FFTPlanDev pl;
  pl.P2 = ctx->P2; pl.Ph = ctx->Ph; pl.M = ctx->M; pl.NM = ctx->NM; pl.Th = ctx->Th; pl.Th2 = ctx->Th2;
  pl.HB = ctx->HB; pl.G = ctx->fftG; pl.lgG = 0;
  while ((1 << pl.lgG) < pl.G) ++pl.lgG;
  pl.tw2 = ctx->d_tw2; pl.twh = ctx->d_twh; pl.thm = ctx->d_thm; pl.bin2c = ctx->d_bin2c;
  return pl;
}

template <class F>
int dispatch_E(int E, F&& f) {
  switch (E) {
    case 3: return f(std::integral_constant<int, 3>());
    case 6: return f(std::integral_constant<int, 6>());
    case 9: return f(std::integral_constant<int, 9>());
    case 12: return f(std::integral_constant<int, 12>());
    case 18: return f(std::integral_constant<int, 18>());
    case 24: return f(std::integral_constant<int, 24>());
  }
  return -1;
}

}  // namespace

// P2 = E G with G the power-of-two part of P2 capped at 32; E must be one of the
// instantiated register-DFT lengths.
bool lsd_fft_plan(lsd_ctx* c) {
  int G = 1;
  while (G < 32 && c->P2 % (2 * G) == 0) G *= 2;
  const int E = c->P2 / G;
  c->fftG = G;
  c->fftE = E;
  return E == 3 || E == 6 || E == 9 || E == 12 || E == 18 || E == 24;
}

int lsd_launch_c2r(lsd_ctx* ctx, const cplx* four, double* phys, int nfields) {
  FFTPlanDev pl = make_plan(ctx);
  dim3 grid(ctx->HB, ctx->N, nfields);
  const size_t smem = sizeof(double2) * 4 * ctx->M + fft_tab_bytes(ctx->fftG, ctx->fftE, ctx->NM);
  int rc = dispatch_E(ctx->fftE, [&](auto e) {
    constexpr int E = decltype(e)::value;
    cudaFuncSetAttribute(k_c2r<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_c2r<E><<<grid, 128, smem, ctx->stream>>>(pl, ctx->N, four, phys);
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
  const size_t smem = sizeof(double2) * 4 * ctx->M + fft_tab_bytes(ctx->fftG, ctx->fftE, ctx->NM);
  int rc = dispatch_E(ctx->fftE, [&](auto e) {
    constexpr int E = decltype(e)::value;
    cudaFuncSetAttribute(k_r2c<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_r2c<E><<<grid, 128, smem, ctx->stream>>>(pl, ctx->N, phys, four);
    return 0;
  });
  if (rc) return lsd_fail(ctx, LSD_EARG, "FFT length not supported");
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_r2c: ") + cudaGetErrorString(e));
  return LSD_OK;
}

int lsd_launch_products(lsd_ctx* ctx, const cplx* four_in, cplx* four_out) {
  FFTPlanDev pl = make_plan(ctx);
  ProdConst pc;
  const lsd_config& c = ctx->cfg;
  pc.d_Cor = 2.0 * c.Pm / c.E;
  pc.Cmag = 2 * c.Pm / c.E;
  pc.d_qm1 = c.Pr / c.Pm;
  pc.sn = ctx->d_sn;
  pc.gp = ctx->d_gp;
  // four rows (a half-row pair) per CTA when they fit, else two (one half-row); then as
  // many staged input fields per round as the sub-groups can take and memory allows
  const size_t budget = 224 * 1024, blk = sizeof(double2) * ctx->M * 4;
  const size_t tabs = fft_tab_bytes(ctx->fftG, ctx->fftE, ctx->NM);
  int RPC = 4;
  size_t fixed = sizeof(double2) * NF_IN * RPC * ctx->P2 + tabs;
  if (fixed + blk > budget) { RPC = 2; fixed = sizeof(double2) * NF_IN * RPC * ctx->P2 + tabs; }
  if (fixed + blk > budget) return lsd_fail(ctx, LSD_EARG, "products: FFT rows do not fit in shared memory");
  const int nsg = 16 * (32 / ctx->fftG);
  int FPR = std::min(NF_IN, nsg / RPC);
  FPR = std::min<int>(FPR, (int)((budget - fixed) / blk));
  const size_t smem = fixed + blk * FPR;
  dim3 grid(RPC == 4 ? ctx->HB : 2 * ctx->HB, ctx->N);
  int rc = dispatch_E(ctx->fftE, [&](auto e) {
    constexpr int E = decltype(e)::value;
    cudaFuncSetAttribute(k_products<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_products<E><<<grid, 512, smem, ctx->stream>>>(pl, ctx->N, pc, four_in, four_out, RPC, FPR);
    return 0;
  });
  if (rc) return lsd_fail(ctx, LSD_EARG, "FFT length not supported");
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_products: ") + cudaGetErrorString(e));
  return LSD_OK;
}
