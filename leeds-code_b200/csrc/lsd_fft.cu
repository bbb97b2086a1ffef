// lsd_fft.cu -- batched real FFTs in phi, standalone and fused with the physical-space
// nonlinear products.
//
// Contract restated from the reference's FFTW use (transform.fftw3.F90:78-93, 280-466):
//  * synthesis (c2r, unnormalised): bins 0..M-1 come from the m-counter map var_Th%m,
//    bins M..Ph/2 are zero, the imaginary part of bin 0 is ignored;
//  * analysis (r2c): input scaled by 1/Ph first, bins 0..M-1 kept, bin 0 exactly real.
// A real transform of length Ph = 2*P2 is done as one complex FFT of length P2 of the
// even/odd-interleaved samples z[t] = x[2t] + i x[2t+1], with the usual split
// pre-/post-processing.  The complex FFT is a shared-memory Stockham autosort with
// radix-4/2/3 passes; P2 = 3M/2 = 3^a 2^b for every supported M.
//
// The fused kernel (one CTA per shell n and TJ theta rows) reads the 15 synthesised
// theta-Fourier rows of u, curl u, B, curl B and grad C, transforms them, forms
//   u x (curl u) + Coriolis + Lorentz      (nonlinear.F90:70-146, Boussinesq)
//   -(Pr/Pm) u . grad C                     (nonlinear.F90:269-272)
//   u x B                                   (nonlinear.F90:421-430)
// at every grid point in shared memory, transforms the 7 results back and writes their
// theta-Fourier rows.  Physical-space fields never touch HBM.
#include "lsd_common.cuh"

namespace {

struct FFTPlanDev {
  int P2, Ph, M, NM, Th, Th2, nrad;
  int rad[16];
  const double2* tw2;  // e^{+2 pi i k/P2}
  const double2* twh;  // e^{+2 pi i k/Ph}
  const int* thm;      // m-counter -> bin
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }

// In-place (ping-pong) Stockham FFT of nrows rows of length P stored contiguously in a
// (row stride P).  sign = +1: e^{+i...} (inverse, unnormalised), -1: forward.
// Returns the buffer holding the result.  All threads of the block must call it.
__device__ double2* block_fft(double2* a, double2* b, int nrows, const FFTPlanDev& pl, int sign) {
  const int P = pl.P2;
  int Ns = 1;
  for (int pass = 0; pass < pl.nrad; ++pass) {
    const int R = pl.rad[pass];
    const int PR = P / R;
    const int tstep = P / (Ns * R);
    const int total = nrows * PR;
    for (int g = threadIdx.x; g < total; g += blockDim.x) {
      const int row = g / PR, t = g - row * PR;
      const int k = t % Ns;
      const double2* src = a + (size_t)row * P;
      double2 v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (q < R) {
          double2 x = src[t + q * PR];
          if (q > 0) {
            double2 w = pl.tw2[(q * k * tstep) % P];
            if (sign < 0) w.y = -w.y;
            x = cmul(x, w);
          }
          v[q] = x;
        }
      }
      double2 o[4];
      if (R == 2) {
        o[0] = make_double2(v[0].x + v[1].x, v[0].y + v[1].y);
        o[1] = make_double2(v[0].x - v[1].x, v[0].y - v[1].y);
      } else if (R == 4) {
        double2 s02 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
        double2 d02 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
        double2 s13 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
        double2 d13 = make_double2(v[1].x - v[3].x, v[1].y - v[3].y);
        // i*sign*d13
        double2 jd13 = sign > 0 ? make_double2(-d13.y, d13.x) : make_double2(d13.y, -d13.x);
        o[0] = make_double2(s02.x + s13.x, s02.y + s13.y);
        o[1] = make_double2(d02.x + jd13.x, d02.y + jd13.y);
        o[2] = make_double2(s02.x - s13.x, s02.y - s13.y);
        o[3] = make_double2(d02.x - jd13.x, d02.y - jd13.y);
      } else {  // R == 3
        const double h = 0.86602540378443864676;  // sqrt(3)/2
        double2 t1 = make_double2(v[1].x + v[2].x, v[1].y + v[2].y);
        double2 t2 = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
        double2 t3 = make_double2(sign * h * (v[1].x - v[2].x), sign * h * (v[1].y - v[2].y));
        o[0] = make_double2(v[0].x + t1.x, v[0].y + t1.y);
        o[1] = make_double2(t2.x - t3.y, t2.y + t3.x);  // t2 + i t3
        o[2] = make_double2(t2.x + t3.y, t2.y - t3.x);  // t2 - i t3
      }
      double2* dst = b + (size_t)row * P;
      const int base = (t / Ns) * Ns * R + k;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (q < R) dst[base + q * Ns] = o[q];
    }
    __syncthreads();
    double2* tmp = a; a = b; b = tmp;
    Ns *= R;
  }
  return a;
}

// Pack the Hermitian half-spectrum Y (bins 0..M-1, rest zero) of one row into the
// half-length complex array Z whose inverse FFT gives z[t] = x[2t] + i x[2t+1].
// Y is read through a lambda ybin(b) returning bin b (b < M) or 0.
template <class YF>
__device__ __forceinline__ double2 c2r_pack(int k, const FFTPlanDev& pl, YF ybin) {
  const int P2 = pl.P2;
  double2 yk = ybin(k);
  double2 yc = conj2(ybin(k == 0 ? P2 : P2 - k));  // conj(Y[P2-k]); Y[P2] = Nyquist = 0
  if (k == 0) yk.y = 0.0;                           // DC imaginary ignored
  double2 s = make_double2(yk.x + yc.x, yk.y + yc.y);
  double2 d = make_double2(yk.x - yc.x, yk.y - yc.y);
  double2 w = pl.twh[k];                            // e^{+2 pi i k/Ph}
  double2 wd = cmul(w, d);
  return make_double2(s.x - wd.y, s.y + wd.x);      // s + i*w*d
}

// From Z = FFT_-(z), bin k < M of the real spectrum (k < P2)
__device__ __forceinline__ double2 r2c_unpack(int k, const double2* Z, const FFTPlanDev& pl) {
  const int P2 = pl.P2;
  double2 zk = Z[k];
  double2 zc = conj2(Z[k == 0 ? 0 : P2 - k]);
  if (k == 0) return make_double2(zk.x + zk.y, 0.0);
  double2 A = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
  double2 Bi = make_double2(0.5 * (zk.x - zc.x), 0.5 * (zk.y - zc.y));  // (Z - conj Z')/2 = i B
  double2 B = make_double2(Bi.y, -Bi.x);                                 // divide by i
  double2 w = conj2(pl.twh[k]);                                          // e^{-2 pi i k/Ph}
  double2 wb = cmul(w, B);
  return make_double2(A.x + wb.x, A.y + wb.y);
}

// The theta-Fourier arrays hold the even/odd half-grid sums of the reference's
// Legendre loops, [f][n][m-counter][p][Th2] with p = 0 (E) and 1 (O): a southern row
// h < Th2 is E + O, its northern mirror Th-1-h is E - O.  A CTA therefore owns TH
// half-rows h and transforms both full rows of each (row 2hh: south, 2hh+1: north);
// for odd Th the equator row is its own mirror and is written once.
__device__ __forceinline__ int row_theta(int h, int side, int Th) { return side ? Th - 1 - h : h; }

// ---- standalone c2r: theta-Fourier -> phys [f][n][Ph][Th] -------------------------------
__global__ void k_c2r(FFTPlanDev pl, int N, const cplx* four, double* phys, int TH) {
  extern __shared__ double2 sm[];
  const int f = blockIdx.z, n = blockIdx.y, h0 = blockIdx.x * TH;
  const int P2 = pl.P2, Th = pl.Th, Th2 = pl.Th2, M = pl.M;
  const int th = min(TH, Th2 - h0);
  const int rows = 2 * th;
  double2* A = sm;
  double2* B = sm + (size_t)2 * TH * P2;
  double2* Ybuf = B;  // bins staged in B first: [row][M]
  const cplx* src = four + ((size_t)f * N + n) * pl.NM * 2 * Th2;
  for (int i = threadIdx.x; i < pl.NM * th; i += blockDim.x) {
    int c = i / th, hh = i % th;
    double2 e = src[((size_t)c * 2 + 0) * Th2 + h0 + hh], o = src[((size_t)c * 2 + 1) * Th2 + h0 + hh];
    int b = pl.thm[c];
    Ybuf[(2 * hh + 0) * M + b] = make_double2(e.x + o.x, e.y + o.y);
    Ybuf[(2 * hh + 1) * M + b] = make_double2(e.x - o.x, e.y - o.y);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < rows * P2; i += blockDim.x) {
    int r = i / P2, k = i % P2;
    const double2* Y = Ybuf + r * M;
    A[r * P2 + k] = c2r_pack(k, pl, [&](int b) { return b < M ? Y[b] : make_double2(0.0, 0.0); });
  }
  __syncthreads();
  double2* R = block_fft(A, B, rows, pl, +1);
  double* dst = phys + ((size_t)f * N + n) * (size_t)pl.Ph * Th;
  for (int i = threadIdx.x; i < rows * P2; i += blockDim.x) {
    int t = i / rows, r = i % rows;
    int hh = r >> 1, side = r & 1, h = h0 + hh;
    int j = row_theta(h, side, Th);
    if (side && j == h) continue;
    double2 z = R[r * P2 + t];
    dst[(size_t)(2 * t) * Th + j] = z.x;
    dst[(size_t)(2 * t + 1) * Th + j] = z.y;
  }
}

// fold two transformed rows (south, north) of half-row h into E and O bins
__device__ __forceinline__ void fold_store(cplx* dst, int c, int Th2, int h, double2 xs, double2 xn, bool equator) {
  double2 e = make_double2(xs.x + xn.x, xs.y + xn.y);
  double2 o = make_double2(xs.x - xn.x, xs.y - xn.y);
  if (equator) { e.x *= 0.5; e.y *= 0.5; }  // odd Th: the equator row is counted once
  dst[((size_t)c * 2 + 0) * Th2 + h] = e;
  dst[((size_t)c * 2 + 1) * Th2 + h] = o;
}

// ---- standalone r2c: phys [f][n][Ph][Th] -> theta-Fourier (folded E/O) ---------------------
__global__ void k_r2c(FFTPlanDev pl, int N, const double* phys, cplx* four, int TH) {
  extern __shared__ double2 sm[];
  const int f = blockIdx.z, n = blockIdx.y, h0 = blockIdx.x * TH;
  const int P2 = pl.P2, Th = pl.Th, Th2 = pl.Th2;
  const int th = min(TH, Th2 - h0);
  const int rows = 2 * th;
  double2* A = sm;
  double2* B = sm + (size_t)2 * TH * P2;
  const double* src = phys + ((size_t)f * N + n) * (size_t)pl.Ph * Th;
  const double scale = 1.0 / (double)pl.Ph;
  for (int i = threadIdx.x; i < rows * P2; i += blockDim.x) {
    int t = i / rows, r = i % rows;
    int j = row_theta(h0 + (r >> 1), r & 1, Th);
    A[r * P2 + t] = make_double2(src[(size_t)(2 * t) * Th + j] * scale, src[(size_t)(2 * t + 1) * Th + j] * scale);
  }
  __syncthreads();
  double2* R = block_fft(A, B, rows, pl, -1);
  cplx* dst = four + ((size_t)f * N + n) * pl.NM * 2 * Th2;
  for (int i = threadIdx.x; i < pl.NM * th; i += blockDim.x) {
    int c = i / th, hh = i % th, h = h0 + hh;
    int b = pl.thm[c];
    double2 xs = r2c_unpack(b, R + (size_t)(2 * hh) * P2, pl);
    double2 xn = r2c_unpack(b, R + (size_t)(2 * hh + 1) * P2, pl);
    fold_store(dst, c, Th2, h, xs, xn, (Th & 1) && h == Th2 - 1);
  }
}

// ---- fused: 15 theta-Fourier inputs -> products -> 7 theta-Fourier outputs -------------
struct ProdConst {
  double d_Cor, Cmag, d_qm1;
  const double* sn;  // sin(theta_j)
  const double* gp;  // cos(theta_j)
};

constexpr int NF_IN = 15, NF_OUT = 7;

__global__ void k_products(FFTPlanDev pl, int N, ProdConst pc, const cplx* four_in, cplx* four_out, int TH) {
  extern __shared__ double2 sm[];
  const int n = blockIdx.y, h0 = blockIdx.x * TH;
  const int P2 = pl.P2, Th = pl.Th, Th2 = pl.Th2, M = pl.M, NM = pl.NM;
  const int th = min(TH, Th2 - h0);
  const int rpf = 2 * th;            // rows per field
  const int rows = NF_IN * rpf;
  double2* A = sm;
  double2* B = sm + (size_t)NF_IN * 2 * TH * P2;
  const size_t fstride = (size_t)N * NM * 2 * Th2;
  // stage bins into B as [row][M], row = f*rpf + 2*hh + side
  for (int i = threadIdx.x; i < NF_IN * NM * th; i += blockDim.x) {
    int hh = i % th, rem = i / th, c = rem % NM, f = rem / NM;
    const cplx* src = four_in + f * fstride + ((size_t)n * NM + c) * 2 * Th2 + h0 + hh;
    double2 e = src[0], o = src[Th2];
    int b = pl.thm[c];
    B[(f * rpf + 2 * hh + 0) * M + b] = make_double2(e.x + o.x, e.y + o.y);
    B[(f * rpf + 2 * hh + 1) * M + b] = make_double2(e.x - o.x, e.y - o.y);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < rows * P2; i += blockDim.x) {
    int row = i / P2, k = i % P2;
    const double2* Y = B + (size_t)row * M;
    A[(size_t)row * P2 + k] = c2r_pack(k, pl, [&](int b) { return b < M ? Y[b] : make_double2(0.0, 0.0); });
  }
  __syncthreads();
  double2* X = block_fft(A, B, rows, pl, +1);
  double2* W = (X == A) ? B : A;  // the other buffer receives the products
  // products at every point (row r, sample t, part re/im)
  for (int i = threadIdx.x; i < rpf * P2; i += blockDim.x) {
    int r = i / P2, t = i % P2;
    int j = row_theta(h0 + (r >> 1), r & 1, Th);
    double sn = pc.sn[j], cs = pc.gp[j];
    double2 v[NF_IN];
#pragma unroll
    for (int f = 0; f < NF_IN; ++f) v[f] = X[(size_t)(f * rpf + r) * P2 + t];
    double2 out[NF_OUT];
#pragma unroll
    for (int part = 0; part < 2; ++part) {
#define G(f) (part == 0 ? v[f].x : v[f].y)
      double vr = G(0), vt = G(1), vp = G(2);
      double wr = G(3), wt = G(4), wp = G(5);
      double br = G(6), bt = G(7), bp = G(8);
      double jr = G(9), jt = G(10), jp = G(11);
      double cr = G(12), ct = G(13), cp = G(14);
#undef G
      double a = vt * wp - vp * wt;
      double b = vp * wr - vr * wp;
      double c = vr * wt - vt * wr;
      a = a + pc.d_Cor * sn * vp;
      b = b + pc.d_Cor * cs * vp;
      c = c - pc.d_Cor * (cs * vt + sn * vr);
      a = a + pc.Cmag * (jt * bp - jp * bt);
      b = b + pc.Cmag * (jp * br - jr * bp);
      c = c + pc.Cmag * (jr * bt - jt * br);
      double e0 = vt * bp - vp * bt;
      double e1 = vp * br - vr * bp;
      double e2 = vr * bt - vt * br;
      double cod = -pc.d_qm1 * vr * cr - pc.d_qm1 * vt * ct - pc.d_qm1 * vp * cp;
      double o[NF_OUT] = {a, b, c, e0, e1, e2, cod};
#pragma unroll
      for (int q = 0; q < NF_OUT; ++q) {
        if (part == 0) out[q].x = o[q]; else out[q].y = o[q];
      }
    }
    const double scale = 1.0 / (double)pl.Ph;
#pragma unroll
    for (int q = 0; q < NF_OUT; ++q)
      W[(size_t)(q * rpf + r) * P2 + t] = make_double2(out[q].x * scale, out[q].y * scale);
  }
  __syncthreads();
  double2* Z = block_fft(W, X, NF_OUT * rpf, pl, -1);
  for (int i = threadIdx.x; i < NF_OUT * NM * th; i += blockDim.x) {
    int hh = i % th, rem = i / th, c = rem % NM, q = rem / NM;
    int h = h0 + hh, b = pl.thm[c];
    double2 xs = r2c_unpack(b, Z + (size_t)(q * rpf + 2 * hh) * P2, pl);
    double2 xn = r2c_unpack(b, Z + (size_t)(q * rpf + 2 * hh + 1) * P2, pl);
    fold_store(four_out + q * fstride + (size_t)n * NM * 2 * Th2, c, Th2, h, xs, xn, (Th & 1) && h == Th2 - 1);
  }
}

FFTPlanDev make_plan(lsd_ctx* ctx) {
  FFTPlanDev pl;
  pl.P2 = ctx->P2; pl.Ph = ctx->Ph; pl.M = ctx->M; pl.NM = ctx->NM; pl.Th = ctx->Th; pl.Th2 = ctx->Th2;
  pl.nrad = ctx->nrad;
  for (int i = 0; i < 16; ++i) pl.rad[i] = ctx->radices[i];
  pl.tw2 = ctx->d_tw2; pl.twh = ctx->d_twh; pl.thm = ctx->d_thm;
  return pl;
}

int pick_tj(int rows_per_j, int P2, size_t budget) {  // half-rows per CTA (2 full rows each)
  size_t per = (size_t)2 * 2 * rows_per_j * P2 * sizeof(double2);
  int tj = (int)(budget / per);
  if (tj > 16) tj = 16;
  return tj < 1 ? 0 : tj;
}

}  // namespace

int lsd_launch_c2r(lsd_ctx* ctx, const cplx* four, double* phys, int nfields) {
  FFTPlanDev pl = make_plan(ctx);
  int TJ = pick_tj(1, ctx->P2, 200 * 1024);
  if (TJ == 0) return lsd_fail(ctx, LSD_EARG, "FFT row does not fit in shared memory");
  size_t smem = (size_t)2 * 2 * TJ * ctx->P2 * sizeof(double2);
  cudaFuncSetAttribute(k_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_c2r, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  dim3 grid(ceil_div(ctx->Th2, TJ), ctx->N, nfields);
  k_c2r<<<grid, 256, smem, ctx->stream>>>(pl, ctx->N, four, phys, TJ);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_c2r: ") + cudaGetErrorString(e));
  return LSD_OK;
}

int lsd_launch_r2c(lsd_ctx* ctx, const double* phys, cplx* four, int nfields) {
  FFTPlanDev pl = make_plan(ctx);
  int TJ = pick_tj(1, ctx->P2, 200 * 1024);
  if (TJ == 0) return lsd_fail(ctx, LSD_EARG, "FFT row does not fit in shared memory");
  size_t smem = (size_t)2 * 2 * TJ * ctx->P2 * sizeof(double2);
  cudaFuncSetAttribute(k_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_r2c, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  dim3 grid(ceil_div(ctx->Th2, TJ), ctx->N, nfields);
  k_r2c<<<grid, 256, smem, ctx->stream>>>(pl, ctx->N, phys, four, TJ);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_r2c: ") + cudaGetErrorString(e));
  return LSD_OK;
}

int lsd_launch_products(lsd_ctx* ctx, const cplx* four_in, cplx* four_out) {
  FFTPlanDev pl = make_plan(ctx);
  int TJ = pick_tj(NF_IN, ctx->P2, 220 * 1024);
  if (TJ == 0) return lsd_fail(ctx, LSD_EARG, "products: FFT rows do not fit in shared memory");
  size_t smem = (size_t)2 * NF_IN * 2 * TJ * ctx->P2 * sizeof(double2);
  // the bin staging area [rows][M] must fit in one buffer
  ProdConst pc;
  const lsd_config& c = ctx->cfg;
  pc.d_Cor = 2.0 * c.Pm / c.E;
  pc.Cmag = 2 * c.Pm / c.E;
  pc.d_qm1 = c.Pr / c.Pm;
  pc.sn = ctx->d_sn;
  pc.gp = ctx->d_gp;
  cudaFuncSetAttribute(k_products, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_products, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  dim3 grid(ceil_div(ctx->Th2, TJ), ctx->N);
  k_products<<<grid, 512, smem, ctx->stream>>>(pl, ctx->N, pc, four_in, four_out, TJ);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_products: ") + cudaGetErrorString(e));
  return LSD_OK;
}
