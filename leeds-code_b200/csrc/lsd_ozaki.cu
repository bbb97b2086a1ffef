// lsd_ozaki.cu -- FP64-accurate Legendre contractions on the tcgen05 tensor cores.
//
// Ozaki-style error-free splitting: an FP64 operand row (or column) is scaled by a power
// of two so that all its entries are below 1 in magnitude, then written as a sum of S
// signed 7-bit digits (int8, |digit| <= 127):  x = 2^e * sum_s d_s 2^(-7(s+1)).
// Products of digit matrices are exact in int32 (|d_a d_b| K <= 127^2 * 256 < 2^31) and
// are accumulated in tensor memory per diagonal s + t; the diagonals s + t < S are
// recombined in FP64 in the epilogue.  The dropped terms bound the relative error by
// about S * K * 2^(-7S) of (row max x column max).
#include <algorithm>
#include <cmath>
#include <vector>

#include "lsd_common.cuh"
#include "lsd_umma.cuh"

namespace {

constexpr long long WAIT_ITERS = 20000000;  // bounded mbarrier polling

// ---- self-test: D(128 x 32) = A(128 x 64) . B(32 x 64)^T in int8 -> int32 ----------------
__global__ void __launch_bounds__(128) k_umma_selftest(const int8_t* A, const int8_t* B, int32_t* D, int* err) {
  __shared__ __align__(1024) int8_t sA[2][128 * 32];
  __shared__ __align__(1024) int8_t sB[2][32 * 32];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < 128 * 64; i += blockDim.x) {
    int r = i / 64, k = i % 64;
    sA[k / 32][umma::tile_off(r, k % 32)] = A[i];
  }
  for (int i = tid; i < 32 * 64; i += blockDim.x) {
    int r = i / 64, k = i % 64;
    sB[k / 32][umma::tile_off(r, k % 32)] = B[i];
  }
  if (tid == 0) umma::mbar_init(&mbar, 1);
  if (warp == 0) umma::tmem_alloc(&tbase, 32);
  umma::fence_proxy_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tbase;
  if (tid == 0) {
    const uint32_t idesc = umma::idesc_s8(128, 32);
    for (int s = 0; s < 2; ++s) {
      uint64_t ad = umma::desc_kmajor_noswz(umma::smem_u32(sA[s]), 128, 256);
      uint64_t bd = umma::desc_kmajor_noswz(umma::smem_u32(sB[s]), 128, 256);
      umma::mma_s8(tmem, ad, bd, idesc, s > 0);
    }
    umma::commit(&mbar);
  }
  __syncwarp();
  bool ok = umma::mbar_wait(&mbar, 0, WAIT_ITERS);
  if (!ok) atomicExch(err, 1);
  umma::fence_after_sync();
  if (ok) {
    for (int c0 = 0; c0 < 32; c0 += 8) {
      int32_t v[8];
      umma::tmem_ld8(tmem + ((uint32_t)(32 * warp) << 16) + c0, v);
      umma::tmem_wait_ld();
      for (int q = 0; q < 8; ++q) D[(32 * warp + (tid & 31)) * 32 + c0 + q] = v[q];
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 32);
}

}  // namespace

// Device self-test of the int8 tensor-core path; *maxerr gets the largest absolute
// difference from the host product (0 when the descriptors and layouts are right).
int lsd_umma_selftest(lsd_ctx* ctx, double* maxerr) {
  std::vector<int8_t> A(128 * 64), B(32 * 64);
  uint32_t s = 12345u;
  auto rnd = [&]() {
    s = s * 1664525u + 1013904223u;
    int v = (int)((s >> 24) & 0xFF) - 128;
    return (int8_t)(v == -128 ? -127 : v);
  };
  for (auto& x : A) x = rnd();
  for (auto& x : B) x = rnd();
  int8_t *dA = nullptr, *dB = nullptr;
  int32_t* dD = nullptr;
  int* dErr = nullptr;
  CUDA_TRY(cudaMalloc(&dA, A.size()));
  CUDA_TRY(cudaMalloc(&dB, B.size()));
  CUDA_TRY(cudaMalloc(&dD, sizeof(int32_t) * 128 * 32));
  CUDA_TRY(cudaMalloc(&dErr, sizeof(int)));
  CUDA_TRY(cudaMemcpy(dA, A.data(), A.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dB, B.data(), B.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemset(dD, 0, sizeof(int32_t) * 128 * 32));
  CUDA_TRY(cudaMemset(dErr, 0, sizeof(int)));
  k_umma_selftest<<<1, 128, 0, ctx->stream>>>(dA, dB, dD, dErr);
  ctx->launches++;
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  std::vector<int32_t> D(128 * 32);
  int err = 0;
  CUDA_TRY(cudaMemcpy(D.data(), dD, sizeof(int32_t) * D.size(), cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(&err, dErr, sizeof(int), cudaMemcpyDeviceToHost));
  cudaFree(dA); cudaFree(dB); cudaFree(dD); cudaFree(dErr);
  if (err) return lsd_fail(ctx, LSD_ECUDA, "tensor-core self-test: mbarrier wait timed out");
  double mx = 0.0;
  for (int m = 0; m < 128; ++m)
    for (int n = 0; n < 32; ++n) {
      long long ref = 0;
      for (int k = 0; k < 64; ++k) ref += (long long)A[m * 64 + k] * B[n * 64 + k];
      mx = std::max(mx, std::fabs((double)(ref - D[m * 32 + n])));
    }
  *maxerr = mx;
  return LSD_OK;
}

// =========================================================================================
// Ozaki Legendre contractions
// =========================================================================================
namespace {

constexpr int OZ_MAXS = 8;      // slices per operand (TMEM: S x 64 columns <= 512)
constexpr int OZ_NC = 32;       // synthesis: theta rows per N chunk

// per (table type, m-counter, parity) GEMM description
struct OzProb {
  int kofs;   // offset of the K-index list (harmonics nh, or theta rows for analysis)
  int len1;   // length of segment 1 (segment 2 follows)
  int K;      // total K
  int nks;    // K steps of 32
  long long bofs;  // byte offset of the table slices
  int fofs;   // offset of the table column exponents
  int npad;   // analysis: N (harmonics) padded to 16; synthesis: theta rows padded to 32
  int nk;     // analysis: number of harmonics of this (counter, parity)
  int nhofs;  // analysis: offset of the harmonic list (nh) of this (counter, parity)
};

// digits of x * 2^-e (|x| < 2^e): S signed 7-bit digits, most significant first
__device__ __forceinline__ void oz_digits(double x, int e, int S, int8_t* d) {
  double y = ldexp(x, -e);
  long long X = (long long)ldexp(y, 7 * S);  // truncation, |X| < 2^(7S)
  long long mag = X < 0 ? -X : X;
  int sgn = X < 0 ? -1 : 1;
#pragma unroll
  for (int s = 0; s < OZ_MAXS; ++s)
    if (s < S) d[s] = (int8_t)(sgn * (int)((mag >> (7 * (S - 1 - s))) & 127));
}

__device__ __forceinline__ int oz_exponent(double maxabs) {
  if (!(maxabs > 0.0)) return -1000;
  int e;
  frexp(maxabs, &e);
  return e;
}

// ---- table slicing at set-up -----------------------------------------------------------
// Synthesis: B(N = theta row j, K = k') with column scale per j.  Tile layout per (chunk of
// 32 rows, K step, slice): 32 x 32 bytes, K-major no swizzle.
struct OzTabArgs {
  const double* leg; int H, Th2, S;
  const OzProb* probs;  // [type][NM][2]
  const int* kidx;
  int8_t* B; int* fexp;
  int tab1[5], tab2[5];  // per type: table of segment 1 / segment 2
  int NM;
};

__global__ void k_oz_slice_synth_tables(OzTabArgs a, int type, int nchunk) {
  const int c = blockIdx.x, p = blockIdx.y;
  const OzProb pr = a.probs[(type * a.NM + c) * 2 + p];
  for (int j = threadIdx.x; j < nchunk * OZ_NC; j += blockDim.x) {
    double mx = 0.0;
    const bool valid = j < a.Th2;
    if (valid)
      for (int k = 0; k < pr.K; ++k) {
        int t = k < pr.len1 ? a.tab1[type] : a.tab2[type];
        double v = a.leg[(size_t)t * a.H * a.Th2 + (size_t)a.kidx[pr.kofs + k] * a.Th2 + j];
        mx = fmax(mx, fabs(v));
      }
    const int e = oz_exponent(mx);
    a.fexp[pr.fofs + j] = e;
    const int ch = j / OZ_NC, r = j % OZ_NC;
    for (int k = 0; k < pr.nks * 32; ++k) {
      int8_t d[OZ_MAXS];
      double v = 0.0;
      if (valid && k < pr.K) {
        int t = k < pr.len1 ? a.tab1[type] : a.tab2[type];
        v = a.leg[(size_t)t * a.H * a.Th2 + (size_t)a.kidx[pr.kofs + k] * a.Th2 + j];
      }
      oz_digits(v, e, a.S, d);
      for (int s = 0; s < a.S; ++s) {
        size_t off = pr.bofs + ((((size_t)ch * pr.nks + k / 32) * a.S + s) * 1024) + umma::tile_off(r, k % 32);
        a.B[off] = d[s];
      }
    }
  }
}

// Analysis: B(N = harmonic k of the (counter, parity), K = theta index j' of the two
// segments) with column scale per k.  Tile per (K step, slice): npad x 32 bytes.
__global__ void k_oz_slice_anal_tables(OzTabArgs a, int type, const int* nhlist) {
  const int c = blockIdx.x, p = blockIdx.y;
  const OzProb pr = a.probs[(type * a.NM + c) * 2 + p];
  for (int k = threadIdx.x; k < pr.npad; k += blockDim.x) {
    const bool valid = k < pr.nk;
    const int nh = valid ? nhlist[pr.nhofs + k] : 0;
    double mx = 0.0;
    if (valid)
      for (int jj = 0; jj < pr.K; ++jj) {
        int t = jj < pr.len1 ? a.tab1[type] : a.tab2[type];
        int j = jj < pr.len1 ? jj : jj - pr.len1;
        mx = fmax(mx, fabs(a.leg[(size_t)t * a.H * a.Th2 + (size_t)nh * a.Th2 + j]));
      }
    const int e = oz_exponent(mx);
    a.fexp[pr.fofs + k] = e;
    for (int jj = 0; jj < pr.nks * 32; ++jj) {
      int8_t d[OZ_MAXS];
      double v = 0.0;
      if (valid && jj < pr.K) {
        int t = jj < pr.len1 ? a.tab1[type] : a.tab2[type];
        int j = jj < pr.len1 ? jj : jj - pr.len1;
        v = a.leg[(size_t)t * a.H * a.Th2 + (size_t)nh * a.Th2 + j];
      }
      oz_digits(v, e, a.S, d);
      for (int s = 0; s < a.S; ++s) {
        size_t off = pr.bofs + (((size_t)(jj / 32) * a.S + s) * (size_t)pr.npad * 32) + umma::tile_off(k, jj % 32);
        a.B[off] = d[s];
      }
    }
  }
}

// ---- data exponents -----------------------------------------------------------------------
// spectral input [n][H]: exponent of max |re|,|im| (times 1/r_n if rinv) over each counter
__global__ void k_oz_exp_spec(int N, int H, int NM, const int* mstart, const int* mlen, const cplx* in,
                              const double* rinv, int* out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  int n = blockIdx.y;
  if (c >= NM) return;
  double mx = 0.0;
  const double r1 = rinv ? rinv[n] : 1.0;
  for (int k = 0; k < mlen[c]; ++k) {
    double2 v = in[(size_t)n * H + mstart[c] + k];
    if (rinv) { v.x *= r1; v.y *= r1; }
    mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
  }
  out[n * NM + c] = oz_exponent(mx);
}
// folded theta-Fourier input [n][c][p][Th2]: exponent of max over p, j
__global__ void k_oz_exp_four(int N, int NM, int Th2, const cplx* in, int* out) {
  int c = blockIdx.x;
  int n = blockIdx.y;
  double mx = 0.0;
  const cplx* src = in + ((size_t)n * NM + c) * 2 * Th2;
  for (int i = threadIdx.x; i < 2 * Th2; i += blockDim.x) mx = fmax(mx, fmax(fabs(src[i].x), fabs(src[i].y)));
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __shared__ double wm[8];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, wm[w]);
    out[n * NM + c] = oz_exponent(mx);
  }
}

// ---- the GEMM kernels ---------------------------------------------------------------------
enum { OZ_VEC = 0, OZ_P = 1, OZ_GRAD = 2 };   // synthesis table types
enum { OZ_ST = 3, OZ_Q = 4 };                 // analysis table types

struct OzSGroup {
  const cplx* in0; const cplx* in1;   // VEC: s, t ; P: q ; GRAD: C
  cplx* out0; cplx* out1;             // VEC/GRAD: theta, phi ; P: r
  const int* e0; const int* e1;       // data exponents [n][NM]
};
struct OzSArgs {
  int N, H, Th2, NM, S, nchunk, nrows, rows_per_group, tmem_cols;
  const OzProb* probs; const int* kidx; const int8_t* B; const int* fexp;
  const double* rinv;
  OzSGroup g[5];
  int* err;
};

// Synthesis GEMM: rows = data (group, shell, component), N = theta rows j (chunks of 32),
// K = harmonics of the counter (two segments).  One CTA: (counter, parity, 128 rows).
template <int TYPE>
__global__ void __launch_bounds__(128, 1) k_oz_synth(OzSArgs a) {
  extern __shared__ __align__(1024) uint8_t oz_smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  __shared__ int fexp_s[OZ_NC];
  const int c = blockIdx.x, p = blockIdx.y;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int S = a.S;
  const OzProb pr = a.probs[(TYPE * a.NM + c) * 2 + p];
  const int nks = pr.nks;
  uint8_t* sA = oz_smem;                                 // [S][nks][4096]
  uint8_t* sB = oz_smem + (size_t)S * nks * 4096;         // [S][nks][1024]
  // ---- the row of this thread and its data
  const int R = blockIdx.z * 128 + tid;
  const bool live = R < a.nrows;
  int g = 0, n = 0, comp = 0;
  if (live) {
    const int per = (TYPE == OZ_P) ? 2 : 4;
    g = R / a.rows_per_group;
    n = (R % a.rows_per_group) / per;
    comp = R % per;
  }
  const OzSGroup G = a.g[g];
  int erow = -1000;
  if (live) {
    if (TYPE == OZ_VEC) erow = max(G.e0[n * a.NM + c], G.e1[n * a.NM + c]);
    else erow = G.e0[n * a.NM + c];
  }
  const double r1 = (TYPE == OZ_GRAD && live) ? a.rinv[n] : 1.0;
  // ---- slice the data rows into A tiles (4 K-bytes at a time per slice)
  for (int k0 = 0; k0 < nks * 32; k0 += 4) {
    uint32_t w[OZ_MAXS];
#pragma unroll
    for (int s = 0; s < OZ_MAXS; ++s) w[s] = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = k0 + u;
      double v = 0.0;
      if (live && k < pr.K) {
        const int nh = a.kidx[pr.kofs + k];
        const bool seg1 = k < pr.len1;
        if (TYPE == OZ_P) {
          double2 q = G.in0[(size_t)n * a.H + nh];
          v = comp ? q.y : q.x;
        } else if (TYPE == OZ_VEC) {
          double2 sv = G.in0[(size_t)n * a.H + nh], tv = G.in1[(size_t)n * a.H + nh];
          if (seg1) v = comp == 0 ? sv.x : comp == 1 ? sv.y : comp == 2 ? tv.x : tv.y;
          else v = comp == 0 ? tv.y : comp == 1 ? -tv.x : comp == 2 ? -sv.y : sv.x;
        } else {  // OZ_GRAD: theta uses P_ (segment 1), phi uses sin1mP (segment 2)
          double2 cv = G.in0[(size_t)n * a.H + nh];
          cv.x *= r1; cv.y *= r1;
          if (seg1) v = comp == 0 ? cv.x : comp == 1 ? cv.y : 0.0;
          else v = comp == 2 ? -cv.y : comp == 3 ? cv.x : 0.0;
        }
      }
      int8_t d[OZ_MAXS];
      oz_digits(v, erow, S, d);
#pragma unroll
      for (int s = 0; s < OZ_MAXS; ++s) w[s] |= ((uint32_t)(uint8_t)d[s]) << (8 * u);
    }
    for (int s = 0; s < S; ++s)
      *(uint32_t*)(sA + ((size_t)s * nks + k0 / 32) * 4096 + umma::tile_off(tid, k0 % 32)) = w[s];
  }
  if (tid == 0) umma::mbar_init(&mbar, 1);
  const uint32_t tcols = a.tmem_cols;
  if (warp == 0) umma::tmem_alloc(&tbase, tcols);
  umma::fence_proxy_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tbase;
  const uint32_t idesc = umma::idesc_s8(128, OZ_NC);
  bool ok = true;
  uint32_t fail_par = 0;
  for (int ch = 0; ch < a.nchunk; ++ch) {
    // ---- table slices of this chunk (copied as 16-byte words)
    const int4* src = (const int4*)(a.B + pr.bofs + (size_t)ch * nks * S * 1024);
    int4* dst = (int4*)sB;
    for (int i = tid; i < nks * S * 64; i += 128) dst[i] = src[i];
    if (tid < OZ_NC) fexp_s[tid] = a.fexp[pr.fofs + ch * OZ_NC + tid];
    umma::fence_proxy_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (tid == 0) {
      for (int ks = 0; ks < nks; ++ks)
        for (int d = 0; d < S; ++d)
          for (int sa = 0; sa <= d; ++sa) {
            const int sb = d - sa;
            uint64_t ad = umma::desc_kmajor_noswz(umma::smem_u32(sA + ((size_t)sa * nks + ks) * 4096), 128, 256);
            uint64_t bd = umma::desc_kmajor_noswz(umma::smem_u32(sB + ((size_t)ks * S + sb) * 1024), 128, 256);
            umma::mma_s8(tmem + (uint32_t)(d * OZ_NC), ad, bd, idesc, (ks > 0 || sa > 0) ? 1 : 0);
          }
      umma::commit(&mbar);
    }
    __syncwarp();
    const bool mine = umma::mbar_wait(&mbar, ch & 1, WAIT_ITERS);
    umma::fence_after_sync();
    if (!__syncthreads_and(mine)) {  // uniform across the CTA
      ok = false;
      fail_par = ch & 1;
      if (tid == 0) atomicExch(a.err, 1);
    }
    if (ok) {
      // ---- epilogue: row tid, 8 theta rows at a time; sum the diagonals from the smallest
      for (int c0 = 0; c0 < OZ_NC; c0 += 8) {
        double acc[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] = 0.0;
        for (int d = S - 1; d >= 0; --d) {
          int32_t v[8];
          umma::tmem_ld8(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(d * OZ_NC + c0), v);
          umma::tmem_wait_ld();
          const double wgt = ldexp(1.0, -7 * (d + 2));
#pragma unroll
          for (int q = 0; q < 8; ++q) acc[q] += (double)v[q] * wgt;
        }
        if (live) {
          cplx* out = (TYPE == OZ_P || comp < 2) ? G.out0 : G.out1;
          double* o = (double*)(out + (((size_t)n * a.NM + c) * 2 + p) * a.Th2) + (comp & 1);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int j = ch * OZ_NC + c0 + q;
            if (j < a.Th2) o[(size_t)j * 2] = ldexp(acc[q], erow + fexp_s[c0 + q]);
          }
        }
      }
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (!ok) break;
  }
  if (!ok) umma::mbar_wait(&mbar, fail_par, WAIT_ITERS);  // error path: let MMAs in flight drain (bounded)
  if (warp == 0) umma::tmem_dealloc(tmem, tcols);
}

struct OzAGroup {
  const cplx* in0; const cplx* in1;   // ST: Y_theta, Y_phi ; Q: Y
  cplx* out0; cplx* out1;             // ST: s, t ; Q: q
  const int* e0; const int* e1;       // data exponents [n][NM]
  int zero_m0_im;                     // Q: zero the imaginary part of m = 0 (scalar analysis)
};
struct OzAArgs {
  int N, H, Th2, NM, S, nrows, rows_per_group, tmem_cols;
  const OzProb* probs; const int* nhlist; const int8_t* B; const int* fexp; const int* hm;
  OzAGroup g[3];
  int* err;
};

// Analysis GEMM: rows = data (group, shell, component), N = harmonics of the (counter,
// parity), K = folded theta rows of the two segments.  Streams K steps through smem.
template <int TYPE>
__global__ void __launch_bounds__(128, 1) k_oz_anal(OzAArgs a) {
  extern __shared__ __align__(1024) uint8_t oz_smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  __shared__ int fexp_s[64];
  __shared__ int nh_s[64];
  const int c = blockIdx.x, p = blockIdx.y;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int S = a.S;
  const OzProb pr = a.probs[(TYPE * a.NM + c) * 2 + p];
  const int npad = pr.npad;
  uint8_t* sA = oz_smem;                    // [S][4096]
  uint8_t* sB = oz_smem + (size_t)S * 4096;  // [S][npad * 32]
  const int R = blockIdx.z * 128 + tid;
  const bool live = R < a.nrows;
  int g = 0, n = 0, comp = 0;
  if (live) {
    const int per = (TYPE == OZ_Q) ? 2 : 4;
    g = R / a.rows_per_group;
    n = (R % a.rows_per_group) / per;
    comp = R % per;
  }
  const OzAGroup G = a.g[g];
  int erow = -1000;
  if (live) erow = (TYPE == OZ_ST) ? max(G.e0[n * a.NM + c], G.e1[n * a.NM + c]) : G.e0[n * a.NM + c];
  if (tid < 64) {
    fexp_s[tid] = tid < npad ? a.fexp[pr.fofs + tid] : 0;
    nh_s[tid] = tid < pr.nk ? a.nhlist[pr.nhofs + tid] : 0;
  }
  if (tid == 0) umma::mbar_init(&mbar, 1);
  const uint32_t tcols = a.tmem_cols;
  if (warp == 0) umma::tmem_alloc(&tbase, tcols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tbase;
  const uint32_t idesc = umma::idesc_s8(128, npad);
  // data pointers of this row: folded E/O rows of the counter at shell n
  const size_t base = ((size_t)n * a.NM + c) * 2 * a.Th2;
  bool ok = true;
  uint32_t fail_par = 0;
  for (int ks = 0; ks < pr.nks; ++ks) {
    for (int k0 = 0; k0 < 32; k0 += 4) {
      uint32_t w[OZ_MAXS];
#pragma unroll
      for (int s = 0; s < OZ_MAXS; ++s) w[s] = 0;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int jj = ks * 32 + k0 + u;
        double v = 0.0;
        if (live && jj < pr.K) {
          if (TYPE == OZ_Q) {
            double2 y = G.in0[base + (size_t)p * a.Th2 + jj];
            v = comp ? y.y : y.x;
          } else {
            const bool seg1 = jj < pr.len1;
            const int j = seg1 ? jj : jj - pr.len1;
            // segment 1 (gwllP_): theta/phi of parity 1-p ; segment 2 (gwllsin1mP): parity p
            const int pp = seg1 ? 1 - p : p;
            double2 yt = G.in0[base + (size_t)pp * a.Th2 + j], yp = G.in1[base + (size_t)pp * a.Th2 + j];
            if (seg1) v = comp == 0 ? yt.x : comp == 1 ? yt.y : comp == 2 ? yp.x : yp.y;
            else v = comp == 0 ? yp.y : comp == 1 ? -yp.x : comp == 2 ? -yt.y : yt.x;
          }
        }
        int8_t d[OZ_MAXS];
        oz_digits(v, erow, S, d);
#pragma unroll
        for (int s = 0; s < OZ_MAXS; ++s) w[s] |= ((uint32_t)(uint8_t)d[s]) << (8 * u);
      }
      for (int s = 0; s < S; ++s) *(uint32_t*)(sA + (size_t)s * 4096 + umma::tile_off(tid, k0)) = w[s];
    }
    const int4* src = (const int4*)(a.B + pr.bofs + (size_t)ks * S * npad * 32);
    int4* dst = (int4*)sB;
    for (int i = tid; i < S * npad * 2; i += 128) dst[i] = src[i];
    umma::fence_proxy_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (tid == 0) {
      for (int d = 0; d < S; ++d)
        for (int sa = 0; sa <= d; ++sa) {
          const int sb = d - sa;
          uint64_t ad = umma::desc_kmajor_noswz(umma::smem_u32(sA + (size_t)sa * 4096), 128, 256);
          uint64_t bd = umma::desc_kmajor_noswz(umma::smem_u32(sB + (size_t)sb * npad * 32), 128, 256);
          umma::mma_s8(tmem + (uint32_t)(d * npad), ad, bd, idesc, (ks > 0 || sa > 0) ? 1 : 0);
        }
      umma::commit(&mbar);
    }
    __syncwarp();
    const bool mine = umma::mbar_wait(&mbar, ks & 1, WAIT_ITERS);
    umma::fence_after_sync();
    if (!__syncthreads_and(mine)) {  // uniform across the CTA
      ok = false;
      fail_par = ks & 1;
      if (tid == 0) atomicExch(a.err, 1);
      break;
    }
  }
  if (ok) {
    for (int c0 = 0; c0 < npad; c0 += 8) {
      double acc[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) acc[q] = 0.0;
      for (int d = S - 1; d >= 0; --d) {
        int32_t v[8];
        umma::tmem_ld8(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(d * npad + c0), v);
        umma::tmem_wait_ld();
        const double wgt = ldexp(1.0, -7 * (d + 2));
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] += (double)v[q] * wgt;
      }
      if (live) {
        cplx* out = (TYPE == OZ_Q || comp < 2) ? G.out0 : G.out1;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int k = c0 + q;
          if (k < pr.nk) {
            const int nh = nh_s[k];
            double val = ldexp(acc[q], erow + fexp_s[k]);
            const bool im = comp & 1;
            // m = 0: s, t (and a scalar) have zero imaginary parts; q keeps its own
            // (transform.fftw3.F90:599, 869, 902, 908)
            if (im && a.hm[nh] == 0 && (TYPE == OZ_ST || G.zero_m0_im)) val = 0.0;
            ((double*)(out + (size_t)n * a.H + nh))[im ? 1 : 0] = val;
          }
        }
      }
    }
  }
  if (!ok) umma::mbar_wait(&mbar, fail_par, WAIT_ITERS);  // error path: let MMAs in flight drain (bounded)
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, tcols);
}

}  // namespace

// =========================================================================================
// host side: set-up of the sliced tables, and the launches
// =========================================================================================
constexpr int OZ_EXP_SLOTS = 32;

struct OzState {
  int S = 0, nchunk = 0, max_nks_synth = 0;
  OzProb* d_probs = nullptr;
  int* d_kidx = nullptr;
  int* d_nh = nullptr;
  int8_t* d_B = nullptr;
  int* d_fexp = nullptr;
  int* d_exp = nullptr;  // data exponents: [slot][N][NM], one slot per input of a launch call
  int* d_err = nullptr;
  std::vector<OzProb> probs;
};

static unsigned pow2cols(int n) {
  unsigned c = 32;
  while ((int)c < n) c <<= 1;
  return c;
}

void lsd_ozaki_free(lsd_ctx* ctx) {
  OzState* o = (OzState*)ctx->oz;
  if (!o) return;
  void* ptrs[] = {o->d_probs, o->d_kidx, o->d_nh, o->d_B, o->d_fexp, o->d_exp, o->d_err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete o;
  ctx->oz = nullptr;
}

int lsd_ozaki_setup(lsd_ctx* ctx) {
  OzState* o = new OzState();
  ctx->oz = o;
  int S = ctx->cfg.ozaki_slices > 0 ? ctx->cfg.ozaki_slices : 7;
  if (S < 2 || S > OZ_MAXS) return lsd_fail(ctx, LSD_EARG, "ozaki_slices must be 2..8");
  o->S = S;
  const int NM = ctx->NM, Th2 = ctx->Th2;
  o->nchunk = ceil_div(Th2, OZ_NC);
  // harmonic lists per (counter, parity)
  std::vector<std::vector<int>> Kcp((size_t)NM * 2);
  for (int c = 0; c < NM; ++c)
    for (int k = 0; k < ctx->mlen[c]; ++k) {
      int nh = ctx->mstart[c] + k;
      Kcp[(size_t)c * 2 + ctx->hs[nh]].push_back(nh);
    }
  std::vector<int> kidx, nhl;
  o->probs.assign((size_t)5 * NM * 2, OzProb());
  long long bytes = 0;
  int fofs = 0;
  for (int type = 0; type < 5; ++type)
    for (int c = 0; c < NM; ++c)
      for (int p = 0; p < 2; ++p) {
        OzProb pr{};
        const std::vector<int>& Kp = Kcp[(size_t)c * 2 + p];
        const std::vector<int>& Kq = Kcp[(size_t)c * 2 + 1 - p];
        pr.nhofs = (int)nhl.size();
        pr.nk = (int)Kp.size();
        nhl.insert(nhl.end(), Kp.begin(), Kp.end());
        pr.kofs = (int)kidx.size();
        if (type == OZ_VEC || type == OZ_GRAD) {  // segment 1 on K(1-p), segment 2 on K(p)
          kidx.insert(kidx.end(), Kq.begin(), Kq.end());
          kidx.insert(kidx.end(), Kp.begin(), Kp.end());
          pr.len1 = (int)Kq.size();
          pr.K = (int)(Kq.size() + Kp.size());
        } else if (type == OZ_P) {
          kidx.insert(kidx.end(), Kp.begin(), Kp.end());
          pr.len1 = pr.K = (int)Kp.size();
        } else if (type == OZ_ST) {
          pr.len1 = Th2;
          pr.K = 2 * Th2;
        } else {
          pr.len1 = pr.K = Th2;
        }
        pr.nks = std::max(1, ceil_div(pr.K, 32));
        pr.bofs = bytes;
        pr.fofs = fofs;
        if (type <= OZ_GRAD) {
          pr.npad = o->nchunk * OZ_NC;
          bytes += (long long)o->nchunk * pr.nks * S * 1024;
          fofs += pr.npad;
          o->max_nks_synth = std::max(o->max_nks_synth, pr.nks);
        } else {
          pr.npad = std::max(16, ((pr.nk + 15) / 16) * 16);
          if (pr.npad > 64) return lsd_fail(ctx, LSD_EARG, "tensor-core analysis supports at most 64 harmonics per (m, parity)");
          bytes += (long long)pr.nks * S * pr.npad * 32;
          fofs += pr.npad;
        }
        o->probs[((size_t)type * NM + c) * 2 + p] = pr;
      }
  size_t smem_synth = std::max((size_t)5120 * S * o->max_nks_synth, (size_t)80 * 1024);
  if (smem_synth > 220 * 1024)
    return lsd_fail(ctx, LSD_EARG, "tensor-core synthesis: too many harmonics per m for the resident slices (reduce ozaki_slices or L)");
  if (kidx.empty()) kidx.push_back(0);
  if (nhl.empty()) nhl.push_back(0);
  CUDA_TRY(cudaMalloc(&o->d_probs, sizeof(OzProb) * o->probs.size()));
  CUDA_TRY(cudaMemcpy(o->d_probs, o->probs.data(), sizeof(OzProb) * o->probs.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMalloc(&o->d_kidx, sizeof(int) * kidx.size()));
  CUDA_TRY(cudaMemcpy(o->d_kidx, kidx.data(), sizeof(int) * kidx.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMalloc(&o->d_nh, sizeof(int) * nhl.size()));
  CUDA_TRY(cudaMemcpy(o->d_nh, nhl.data(), sizeof(int) * nhl.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMalloc(&o->d_B, bytes));
  CUDA_TRY(cudaMalloc(&o->d_fexp, sizeof(int) * (size_t)fofs));
  CUDA_TRY(cudaMalloc(&o->d_exp, sizeof(int) * (size_t)OZ_EXP_SLOTS * ctx->N * NM));
  CUDA_TRY(cudaMalloc(&o->d_err, sizeof(int)));
  CUDA_TRY(cudaMemset(o->d_err, 0, sizeof(int)));
  OzTabArgs ta;
  ta.leg = ctx->d_leg; ta.H = ctx->H; ta.Th2 = Th2; ta.S = S; ta.probs = o->d_probs; ta.kidx = o->d_kidx;
  ta.B = o->d_B; ta.fexp = o->d_fexp; ta.NM = NM;
  const int t1[5] = {LSD_LEG_LLP_, LSD_LEG_P, LSD_LEG_P_, LSD_LEG_GWLLP_, LSD_LEG_GWP};
  const int t2[5] = {LSD_LEG_LLSIN1MP, LSD_LEG_P, LSD_LEG_SIN1MP, LSD_LEG_GWLLSIN1MP, LSD_LEG_GWP};
  for (int i = 0; i < 5; ++i) { ta.tab1[i] = t1[i]; ta.tab2[i] = t2[i]; }
  dim3 g(NM, 2);
  for (int type = 0; type <= OZ_GRAD; ++type) k_oz_slice_synth_tables<<<g, 128, 0, ctx->stream>>>(ta, type, o->nchunk);
  for (int type = OZ_ST; type <= OZ_Q; ++type) k_oz_slice_anal_tables<<<g, 64, 0, ctx->stream>>>(ta, type, o->d_nh);
  ctx->launches += 5;
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (int type = 0; type <= OZ_GRAD; ++type) {
    auto kern = type == OZ_VEC ? k_oz_synth<OZ_VEC> : type == OZ_P ? k_oz_synth<OZ_P> : k_oz_synth<OZ_GRAD>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_synth);
  }
  return LSD_OK;
}

// data exponents of a spectral input (slot < 14) or a theta-Fourier input (slot 14..20)
static int oz_exp_spec(lsd_ctx* ctx, const cplx* in, const double* rinv, int slot) {
  OzState* o = (OzState*)ctx->oz;
  dim3 g(ceil_div(ctx->NM, 64), ctx->N);
  k_oz_exp_spec<<<g, 64, 0, ctx->stream>>>(ctx->N, ctx->H, ctx->NM, ctx->d_mstart, ctx->d_mlen, in, rinv,
                                            o->d_exp + (size_t)slot * ctx->N * ctx->NM);
  ctx->launches++;
  return LSD_OK;
}
static int oz_exp_four(lsd_ctx* ctx, const cplx* in, int slot) {
  OzState* o = (OzState*)ctx->oz;
  dim3 g(ctx->NM, ctx->N);
  k_oz_exp_four<<<g, 128, 0, ctx->stream>>>(ctx->N, ctx->NM, ctx->Th2, in, o->d_exp + (size_t)slot * ctx->N * ctx->NM);
  ctx->launches++;
  return LSD_OK;
}

const int* lsd_ozaki_exp(lsd_ctx* ctx, int slot) {
  OzState* o = (OzState*)ctx->oz;
  return o->d_exp + (size_t)slot * ctx->N * ctx->NM;
}
int lsd_ozaki_exp_spec(lsd_ctx* ctx, const cplx* in, const double* rinv, int slot) { return oz_exp_spec(ctx, in, rinv, slot); }
int lsd_ozaki_exp_four(lsd_ctx* ctx, const cplx* in, int slot) { return oz_exp_four(ctx, in, slot); }

// groups: VEC {s, t -> theta, phi}, P {q -> r}, GRAD {C -> theta, phi}
int lsd_ozaki_synth(lsd_ctx* ctx, int type, const OzSynthGroupH* gh, int ng) {
  OzState* o = (OzState*)ctx->oz;
  OzSArgs a;
  a.N = ctx->N; a.H = ctx->H; a.Th2 = ctx->Th2; a.NM = ctx->NM; a.S = o->S; a.nchunk = o->nchunk;
  const int per = (type == OZ_P) ? 2 : 4;
  a.rows_per_group = per * ctx->N;
  a.nrows = ng * a.rows_per_group;
  a.tmem_cols = pow2cols(o->S * OZ_NC);
  a.probs = o->d_probs; a.kidx = o->d_kidx; a.B = o->d_B; a.fexp = o->d_fexp;
  a.rinv = ctx->d_r + (size_t)2 * ctx->N;
  a.err = o->d_err;
  for (int i = 0; i < ng; ++i) {
    a.g[i].in0 = gh[i].in0; a.g[i].in1 = gh[i].in1; a.g[i].out0 = gh[i].out0; a.g[i].out1 = gh[i].out1;
    a.g[i].e0 = gh[i].e0; a.g[i].e1 = gh[i].e1;
  }
  dim3 grid(ctx->NM, 2, ceil_div(a.nrows, 128));
  // at most two CTAs (2 x 256 TMEM columns) per SM
  size_t smem = std::max((size_t)5120 * o->S * o->max_nks_synth, (size_t)80 * 1024);
  if (type == OZ_VEC) k_oz_synth<OZ_VEC><<<grid, 128, smem, ctx->stream>>>(a);
  else if (type == OZ_P) k_oz_synth<OZ_P><<<grid, 128, smem, ctx->stream>>>(a);
  else k_oz_synth<OZ_GRAD><<<grid, 128, smem, ctx->stream>>>(a);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_oz_synth: ") + cudaGetErrorString(e));
  return LSD_OK;
}

// groups: ST {Y_theta, Y_phi -> s, t}, Q {Y -> q}
int lsd_ozaki_anal(lsd_ctx* ctx, int type, const OzAnalGroupH* gh, int ng) {
  OzState* o = (OzState*)ctx->oz;
  OzAArgs a;
  a.N = ctx->N; a.H = ctx->H; a.Th2 = ctx->Th2; a.NM = ctx->NM; a.S = o->S;
  const int per = (type == OZ_Q) ? 2 : 4;
  a.rows_per_group = per * ctx->N;
  a.nrows = ng * a.rows_per_group;
  a.tmem_cols = pow2cols(o->S * 64);
  a.probs = o->d_probs; a.nhlist = o->d_nh; a.B = o->d_B; a.fexp = o->d_fexp; a.hm = ctx->d_m;
  a.err = o->d_err;
  for (int i = 0; i < ng; ++i) {
    a.g[i].in0 = gh[i].in0; a.g[i].in1 = gh[i].in1; a.g[i].out0 = gh[i].out0; a.g[i].out1 = gh[i].out1;
    a.g[i].e0 = gh[i].e0; a.g[i].e1 = gh[i].e1; a.g[i].zero_m0_im = gh[i].zero_m0_im;
  }
  dim3 grid(ctx->NM, 2, ceil_div(a.nrows, 128));
  size_t smem = (size_t)o->S * (4096 + 64 * 32) + 1024;
  // ask for more than half of an SM's shared memory: one CTA (one TMEM allocation) per SM
  smem = std::max(smem, (size_t)120 * 1024);
  if (type == OZ_ST) {
    cudaFuncSetAttribute(k_oz_anal<OZ_ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_oz_anal<OZ_ST><<<grid, 128, smem, ctx->stream>>>(a);
  } else {
    cudaFuncSetAttribute(k_oz_anal<OZ_Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_oz_anal<OZ_Q><<<grid, 128, smem, ctx->stream>>>(a);
  }
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_oz_anal: ") + cudaGetErrorString(e));
  return LSD_OK;
}

int* lsd_ozaki_err_flag(lsd_ctx* ctx) { return ((OzState*)ctx->oz)->d_err; }

int lsd_ozaki_check(lsd_ctx* ctx) {
  OzState* o = (OzState*)ctx->oz;
  int err = 0;
  CUDA_TRY(cudaMemcpy(&err, o->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return lsd_fail(ctx, LSD_ECUDA, "tensor-core contraction: an mbarrier wait timed out");
  return LSD_OK;
}

// The FP64 group descriptions of the synthesis / analysis launchers, mapped onto the
// tensor-core GEMM types: vector (q,s,t) = P(q) + VEC(s,t); scalar = P; grad3 (dC, C) =
// P(dC) + GRAD(C); grad2 = GRAD; analysis vector (r,th,ph) = Q(r) + ST(th,ph); scalar = Q.
int lsd_ozaki_launch_synth(lsd_ctx* ctx, const SynthGroup* groups, int ngroups) {
  OzState* o = (OzState*)ctx->oz;
  const double* rinv = ctx->d_r + (size_t)2 * ctx->N;
  std::vector<OzSynthGroupH> gv, gp, gg;
  int slot = 0;
  auto ex = [&](const cplx* in, const double* ri) -> const int* {
    if (slot >= OZ_EXP_SLOTS) return nullptr;
    oz_exp_spec(ctx, in, ri, slot);
    return o->d_exp + (size_t)(slot++) * ctx->N * ctx->NM;
  };
  for (int i = 0; i < ngroups; ++i) {
    const SynthGroup& G = groups[i];
    OzSynthGroupH h{};
    switch (G.kind) {
      case SK_VECTOR:
        h = {G.in[0], nullptr, G.out[0], nullptr, ex(G.in[0], nullptr), nullptr};
        gp.push_back(h);
        h = {G.in[1], G.in[2], G.out[1], G.out[2], ex(G.in[1], nullptr), ex(G.in[2], nullptr)};
        gv.push_back(h);
        break;
      case SK_SCALAR:
        h = {G.in[0], nullptr, G.out[0], nullptr, ex(G.in[0], nullptr), nullptr};
        gp.push_back(h);
        break;
      case SK_GRAD3:
        h = {G.in[0], nullptr, G.out[0], nullptr, ex(G.in[0], nullptr), nullptr};
        gp.push_back(h);
        h = {G.in[1], nullptr, G.out[1], G.out[2], ex(G.in[1], rinv), nullptr};
        gg.push_back(h);
        break;
      default:  // SK_GRAD2
        h = {G.in[0], nullptr, G.out[0], G.out[1], ex(G.in[0], rinv), nullptr};
        gg.push_back(h);
        break;
    }
  }
  if (slot >= OZ_EXP_SLOTS) return lsd_fail(ctx, LSD_EARG, "tensor-core synthesis: too many inputs in one call");
  int rc;
  for (size_t i = 0; i < gv.size(); i += 5)
    if ((rc = lsd_ozaki_synth(ctx, OZ_VEC, gv.data() + i, (int)std::min<size_t>(5, gv.size() - i)))) return rc;
  for (size_t i = 0; i < gp.size(); i += 5)
    if ((rc = lsd_ozaki_synth(ctx, OZ_P, gp.data() + i, (int)std::min<size_t>(5, gp.size() - i)))) return rc;
  for (size_t i = 0; i < gg.size(); i += 5)
    if ((rc = lsd_ozaki_synth(ctx, OZ_GRAD, gg.data() + i, (int)std::min<size_t>(5, gg.size() - i)))) return rc;
  return LSD_OK;
}

int lsd_ozaki_launch_anal(lsd_ctx* ctx, const AnalGroup* groups, int ngroups) {
  OzState* o = (OzState*)ctx->oz;
  std::vector<OzAnalGroupH> gs, gq;
  int slot = 0;
  auto ex = [&](const cplx* in) -> const int* {
    if (slot >= OZ_EXP_SLOTS) return nullptr;
    oz_exp_four(ctx, in, slot);
    return o->d_exp + (size_t)(slot++) * ctx->N * ctx->NM;
  };
  for (int i = 0; i < ngroups; ++i) {
    const AnalGroup& G = groups[i];
    OzAnalGroupH h{};
    if (G.kind == AK_VECTOR) {
      h = {G.in[0], nullptr, G.out[0], nullptr, ex(G.in[0]), nullptr, 0};  // q keeps Im of m = 0
      gq.push_back(h);
      h = {G.in[1], G.in[2], G.out[1], G.out[2], ex(G.in[1]), ex(G.in[2]), 1};
      gs.push_back(h);
    } else {
      h = {G.in[0], nullptr, G.out[0], nullptr, ex(G.in[0]), nullptr, 1};
      gq.push_back(h);
    }
  }
  if (slot >= OZ_EXP_SLOTS) return lsd_fail(ctx, LSD_EARG, "tensor-core analysis: too many inputs in one call");
  int rc;
  for (size_t i = 0; i < gs.size(); i += 3)
    if ((rc = lsd_ozaki_anal(ctx, OZ_ST, gs.data() + i, (int)std::min<size_t>(3, gs.size() - i)))) return rc;
  for (size_t i = 0; i < gq.size(); i += 3)
    if ((rc = lsd_ozaki_anal(ctx, OZ_Q, gq.data() + i, (int)std::min<size_t>(3, gq.size() - i)))) return rc;
  return LSD_OK;
}
