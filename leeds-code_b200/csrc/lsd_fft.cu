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

// Inverse (e^{+i}) FFT of length E*G.  In: v[k1] = Z[k1 + E l].  Out: v[e] = x[brev(l) + G e].
template <int E>
__device__ __forceinline__ void wfft_inv(double2 (&v)[E], int l, const FFTPlanDev& pl) {
  const int G = pl.G;
  for (int h = G >> 1; h >= 1; h >>= 1) {  // radix-2 DIF over the lanes (natural -> bit-reversed)
    const bool up = l & h;
    const double2 w = __ldg(&pl.tw2[E * (l & (h - 1)) * (G / (2 * h))]);
#pragma unroll
    for (int k = 0; k < E; ++k) {
      const double2 p = shfl_xor2(v[k], h);
      v[k] = up ? cmul(sub2(p, v[k]), w) : add2(v[k], p);
    }
  }
  const int g = brev_bits(l, pl.lgG);
#pragma unroll
  for (int k = 1; k < E; ++k) v[k] = cmul(v[k], __ldg(&pl.tw2[g * k]));
  double2 x[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {  // E-point DFT in registers, w_E = w_P2^G
    double2 s = v[0];
#pragma unroll
    for (int k = 1; k < E; ++k) s = add2(s, cmul(v[k], __ldg(&pl.tw2[G * ((e * k) % E)])));
    x[e] = s;
  }
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = x[e];
}

// Forward (e^{-i}) FFT, the mirror of wfft_inv.  In: v[e] = x[brev(l) + G e].
// Out: v[k1] = X[k1 + E l].
template <int E>
__device__ __forceinline__ void wfft_fwd(double2 (&v)[E], int l, const FFTPlanDev& pl) {
  const int G = pl.G;
  double2 u[E];
#pragma unroll
  for (int k = 0; k < E; ++k) {
    double2 s = v[0];
#pragma unroll
    for (int e = 1; e < E; ++e) s = add2(s, cmulc(v[e], __ldg(&pl.tw2[G * ((e * k) % E)])));
    u[k] = s;
  }
  const int g = brev_bits(l, pl.lgG);
#pragma unroll
  for (int k = 0; k < E; ++k) v[k] = k ? cmulc(u[k], __ldg(&pl.tw2[g * k])) : u[0];
  for (int h = 1; h < G; h <<= 1) {  // radix-2 DIT over the lanes (bit-reversed -> natural)
    const bool up = l & h;
    const double2 w = __ldg(&pl.tw2[E * (l & (h - 1)) * (G / (2 * h))]);
#pragma unroll
    for (int k = 0; k < E; ++k) {
      const double2 send = up ? cmulc(v[k], w) : v[k];
      const double2 recv = shfl_xor2(send, h);
      v[k] = up ? sub2(recv, send) : add2(send, recv);
    }
  }
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

// Spectrum Y[b] of one full theta row from the folded rows of counter bin2c[b] in a
// half-row-pair block: south E + O, north E - O.
__device__ __forceinline__ double2 row_bin(const cplx* blk, int b, int jj, int side, const FFTPlanDev& pl) {
  if (b >= pl.M) return make_double2(0.0, 0.0);
  const int c = __ldg(&pl.bin2c[b]);
  const double2 e = __ldg(&blk[(c * 2 + 0) * 2 + jj]), o = __ldg(&blk[(c * 2 + 1) * 2 + jj]);
  return side ? sub2(e, o) : add2(e, o);
}

// Load + pack + inverse FFT of one row; blk = the (n, h/2) block of one field.
template <int E>
__device__ __forceinline__ void row_c2r(double2 (&v)[E], const cplx* blk, int jj, int side, int l, const FFTPlanDev& pl) {
  const int P2 = pl.P2;
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) {
    const int k = k1 + E * l;
    v[k1] = c2r_pack(k, row_bin(blk, k, jj, side, pl), row_bin(blk, k == 0 ? P2 : P2 - k, jj, side, pl), pl);
  }
  wfft_inv<E>(v, l, pl);
}

// Forward FFT of one row of physical samples (lane order) + unpack of bins b = k1 + E l.
// The partner Z[P2 - k] lives in lane (G - l) % G (k1 = 0) or G - 1 - l (register E - k1).
template <int E>
__device__ __forceinline__ void row_r2c(double2 (&v)[E], int l, int lane0, const FFTPlanDev& pl) {
  const int G = pl.G;
  wfft_fwd<E>(v, l, pl);
  double2 out[E];
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) {
    const int src = k1 == 0 ? (G - l) % G : G - 1 - l;
    const double2 zm = shfl2(v[k1 == 0 ? 0 : E - k1], lane0 + src);
    out[k1] = r2c_unpack(k1 + E * l, v[k1], zm, pl);
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
// blockIdx.x = h, for long rows).  smem: [NF_IN][RPC][P2] double2.
template <int E>
__global__ void __launch_bounds__(512) k_products(FFTPlanDev pl, int N, ProdConst pc, const cplx* four_in,
                                                  cplx* four_out, int RPC) {
  extern __shared__ double2 phys[];
  const int n = blockIdx.y;
  const int hb = RPC == 4 ? blockIdx.x : blockIdx.x >> 1;
  const int jj0 = RPC == 4 ? 0 : (blockIdx.x & 1);
  const int P2 = pl.P2, G = pl.G, NM = pl.NM, Th = pl.Th, Th2 = pl.Th2;
  const size_t fstride = (size_t)N * pl.HB * NM * 4;
  const size_t boff = ((size_t)n * pl.HB + hb) * NM * 4;  // the CTA's block in every field
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int sgw = 32 / G, l = lane % G, lane0 = lane - l;
  // ---- inverse transforms: task = (field, row), G lanes per task
  for (int t0 = warp * sgw; t0 < NF_IN * RPC; t0 += nw * sgw) {
    const int t = t0 + lane / G;
    const int tt = t < NF_IN * RPC ? t : t0;  // lanes without a task redo a valid one
    const int f = tt / RPC, r = tt % RPC;
    const int jj = jj0 + (r >> 1), side = r & 1;
    const bool act = t < NF_IN * RPC && 2 * hb + jj < Th2;
    double2 v[E];
    row_c2r<E>(v, four_in + f * fstride + boff, jj, side, l, pl);
    if (act) {
      double2* dst = phys + ((size_t)f * RPC + r) * P2;
#pragma unroll
      for (int e = 0; e < E; ++e) dst[e * G + l] = v[e];
    }
  }
  __syncthreads();
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
    const int tt = t < NF_OUT * RPC ? t : t0;
    const int q = tt / RPC, r = tt % RPC;
    const bool act = t < NF_OUT * RPC && 2 * hb + jj0 + (r >> 1) < Th2;
    double2* slot = phys + ((size_t)q * RPC + r) * P2;
    double2 v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = slot[e * G + l];
    row_r2c<E>(v, l, lane0, pl);
    __syncwarp();
    if (act) {
#pragma unroll
      for (int k1 = 0; k1 < E; ++k1) {
        const int b = k1 + E * l;
        if (b < pl.M) slot[b] = v[k1];
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
    const int b = pl.thm[c];
    const double2 xs = phys[((size_t)q * RPC + 2 * jr) * P2 + b];
    const double2 xn = phys[((size_t)q * RPC + 2 * jr + 1) * P2 + b];
    double2 val = p == 0 ? add2(xs, xn) : sub2(xs, xn);
    if (p == 0 && (Th & 1) && h == Th2 - 1) { val.x *= 0.5; val.y *= 0.5; }  // odd Th: equator once
    four_out[q * fstride + boff + (c * 2 + p) * 2 + jj] = val;
  }
}

// ---- standalone c2r: theta-Fourier -> phys [f][n][Ph][Th] -------------------------------
// grid (Th2, N, nfields), 64 threads: the two theta rows of half-row h, G lanes each.
template <int E>
__global__ void __launch_bounds__(64) k_c2r(FFTPlanDev pl, int N, const cplx* four, double* phys) {
  const int h = blockIdx.x, n = blockIdx.y, f = blockIdx.z;
  const int G = pl.G, Th = pl.Th;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int l = lane % G;
  const int grp = warp * (32 / G) + lane / G;  // groups 0, 1 take the rows; others redo row 0
  const int side = grp & 1;
  const cplx* blk = four + (((size_t)f * N + n) * pl.HB + (h >> 1)) * pl.NM * 4;
  double2 v[E];
  row_c2r<E>(v, blk, h & 1, side, l, pl);
  const int j = row_theta(h, side, Th);
  if (grp > 1 || (side && j == h)) return;  // odd Th: the equator row is written once
  double* dst = phys + ((size_t)f * N + n) * (size_t)pl.Ph * Th;
  const int g = brev_bits(l, pl.lgG);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int t = g + G * e;
    dst[(size_t)(2 * t) * Th + j] = v[e].x;
    dst[(size_t)(2 * t + 1) * Th + j] = v[e].y;
  }
}

// ---- standalone r2c: phys [f][n][Ph][Th] -> folded theta-Fourier --------------------------
template <int E>
__global__ void __launch_bounds__(64) k_r2c(FFTPlanDev pl, int N, const double* phys, cplx* four) {
  __shared__ double2 bins[2][512];
  const int h = blockIdx.x, n = blockIdx.y, f = blockIdx.z;
  const int G = pl.G, Th = pl.Th, Th2 = pl.Th2, M = pl.M;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int l = lane % G, lane0 = lane - l;
  const int grp = warp * (32 / G) + lane / G;
  const int side = grp & 1;
  const double scale = 1.0 / (double)pl.Ph;
  const int j = row_theta(h, side, Th);
  const double* src = phys + ((size_t)f * N + n) * (size_t)pl.Ph * Th;
  const int g = brev_bits(l, pl.lgG);
  double2 v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int t = g + G * e;
    v[e] = make_double2(src[(size_t)(2 * t) * Th + j] * scale, src[(size_t)(2 * t + 1) * Th + j] * scale);
  }
  row_r2c<E>(v, l, lane0, pl);
  if (grp <= 1) {
#pragma unroll
    for (int k1 = 0; k1 < E; ++k1) {
      const int b = k1 + E * l;
      if (b < M) bins[side][b] = v[k1];
    }
  }
  __syncthreads();
  cplx* blk = four + (((size_t)f * N + n) * pl.HB + (h >> 1)) * pl.NM * 4;
  for (int i = threadIdx.x; i < pl.NM * 2; i += blockDim.x) {
    const int c = i >> 1, p = i & 1, b = pl.thm[c];
    double2 val = p == 0 ? add2(bins[0][b], bins[1][b]) : sub2(bins[0][b], bins[1][b]);
    if (p == 0 && (Th & 1) && h == Th2 - 1) { val.x *= 0.5; val.y *= 0.5; }
    blk[(c * 2 + p) * 2 + (h & 1)] = val;
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
  dim3 grid(ctx->Th2, ctx->N, nfields);
  int rc = dispatch_E(ctx->fftE, [&](auto e) {
    k_c2r<decltype(e)::value><<<grid, 64, 0, ctx->stream>>>(pl, ctx->N, four, phys);
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
  if (ctx->M > 512) return lsd_fail(ctx, LSD_EARG, "r2c: more than 512 bins");
  dim3 grid(ctx->Th2, ctx->N, nfields);
  int rc = dispatch_E(ctx->fftE, [&](auto e) {
    k_r2c<decltype(e)::value><<<grid, 64, 0, ctx->stream>>>(pl, ctx->N, phys, four);
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
  // four rows (a half-row pair) per CTA when they fit, else two (one half-row)
  int RPC = 4;
  size_t smem = sizeof(double2) * NF_IN * RPC * ctx->P2;
  if (smem > 220 * 1024) { RPC = 2; smem /= 2; }
  if (smem > 220 * 1024) return lsd_fail(ctx, LSD_EARG, "products: FFT rows do not fit in shared memory");
  dim3 grid(RPC == 4 ? ctx->HB : 2 * ctx->HB, ctx->N);
  int rc = dispatch_E(ctx->fftE, [&](auto e) {
    constexpr int E = decltype(e)::value;
    cudaFuncSetAttribute(k_products<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_products<E><<<grid, 512, smem, ctx->stream>>>(pl, ctx->N, pc, four_in, four_out, RPC);
    return 0;
  });
  if (rc) return lsd_fail(ctx, LSD_EARG, "FFT length not supported");
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_products: ") + cudaGetErrorString(e));
  return LSD_OK;
}
