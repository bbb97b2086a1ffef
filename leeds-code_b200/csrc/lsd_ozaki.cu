// lsd_ozaki.cu -- FP64-accurate Legendre contractions on the tcgen05 tensor cores.
//
// Ozaki-style splitting: an FP64 operand row (or column) with entries below 2^e in
// magnitude is rounded to the nearest integer X of x 2^(8S - 2 - e) (|X| < 2^(8S-2)) and
// X is written as S balanced base-256 digits, int8 in [-128, 127]:
//   x ~= 2^(e+2) * sum_s d_s 2^(-8(s+1)),  s = 0 most significant.
// The digits are the bytes of X + C, C = 0x80 in every byte below the top one, with bit 7
// of those lower bytes flipped (b - 128); the top byte of X + C is the top digit as it is
// (|d_0| <= 65).  Rounding to nearest keeps the error unbiased, and the digits come out of
// the integer by byte permutes alone.  Products of digit matrices are exact in int32
// (S K 128^2 < 2^31 for K <= 16384) and are accumulated in tensor memory per diagonal
// s + t; the diagonals s + t < S are recombined in FP64 in the epilogue.  Per product the
// rounding costs 2^(1-8S) and the dropped diagonals about (S + 1) 2^(2-8S) of
// (row max x column max).
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
  // on the context's stream, which the kernel below runs on (a plain cudaMemcpy from
  // pageable memory may return before its DMA lands, and is not ordered with that stream)
  CUDA_TRY(cudaMemcpyAsync(dA, A.data(), A.size(), cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaMemcpyAsync(dB, B.data(), B.size(), cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaMemsetAsync(dD, 0, sizeof(int32_t) * 128 * 32, ctx->stream));
  CUDA_TRY(cudaMemsetAsync(dErr, 0, sizeof(int), ctx->stream));
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
//
// Every contraction of one m-counter c and one output parity p is a real GEMM
//   D[row, col] = sum_k A[row, k] B[k, col]
// rows: the data (group, shell, component re/im of the inputs), 128 per CTA ("z-block");
// columns: theta rows j of the half grid (synthesis) or the harmonics of (c, p) (analysis),
// NC per chunk (48 or 32, oz_nc); k: harmonics of c in two segments (synthesis) or the folded theta rows of
// two parities (analysis), 32 per K step.  The sign/parity recipes of the reference's
// accumulations (transform.fftw3.F90:746-774, 866-909) are folded into the A rows.
//
// Two kernels per contraction: a slicing pre-pass reads the FP64 data once, takes each
// row's exponent and writes the int8 digits in the tcgen05 shared-memory tile layout; the
// GEMM streams A and B tiles with bulk copies (a ring of 2-4 stages), issues the int8 MMAs of
// the S(S+1)/2 digit pairs into S tensor-memory diagonals, and its epilogue warps read the
// diagonals into registers, hand the tensor memory back, recombine them exactly and store
// straight to HBM.
// =========================================================================================
namespace {

constexpr int OZ_MAXS = 8;       // slices per operand
constexpr int OZ_NCMAX = 48;     // columns per chunk: 48 or 32 (oz_nc)
constexpr int OZ_MAXSTAGES = 4;  // bulk-copy ring: up to 4 stages (default 3 where two CTAs per SM fit)
constexpr int OZ_EPI = 256;      // epilogue threads: warps 0-7 (warp w: TMEM lane quarter w % 4,
                                 // column half w / 4 of a chunk)
constexpr int OZ_THREADS = OZ_EPI + 64;  // + warp 8 (bulk copies) and warp 9 (MMA issue)
constexpr int OZ_MAXG = 8;       // groups (output fields) of one launch

enum { OZ_VEC = 0, OZ_P = 1, OZ_GRAD = 2, OZ_ST = 3, OZ_Q = 4, OZ_NTYPE = 5 };

// Columns per chunk: 48 for the synthesis types while the S diagonals of a chunk fit the
// CTA's 256 tensor-memory columns (S <= 5; theta rows come in multiples of 48 at lmax 127
// and 255, and the largest MMA is N = 240), else 32; the analysis types keep 32 (their
// columns are the <= 64 harmonics of one (m, parity)).  Fewer, wider MMAs per K step.
__host__ __device__ constexpr int oz_nc(int type, int S) { return type < OZ_ST && S * 48 <= 256 ? 48 : 32; }
// bytes of one ring stage (A: S x 4096, B: S slices of NC x 32), the widest chunk's
constexpr size_t oz_stage_bytes(int S) { return (size_t)S * (4096 + oz_nc(OZ_VEC, S) * 32); }

// per (type, m-counter, parity)
struct OzProb {
  int kofs;        // synthesis: offset of the K list (harmonics nh)
  int len1;        // K length of segment 1 (segment 2 follows)
  int K;           // total K
  int nks;         // K steps of 32
  int nchunk;      // column chunks of 32
  int nk;          // analysis: harmonics of (c, p)
  int nhofs;       // analysis: offset of their list
  int fofs;        // column exponents (nchunk * 32)
  long long bofs;  // table digits [chunk][ks][slice][32 x 32]
  long long aofs;  // data digits of z-block 0 [zb][ks][slice][128 x 32]
};

// 2^e exactly (bit construction in the normal range)
__device__ __forceinline__ double pow2i(int e) {
  if (e >= -1022 && e <= 1023) return __longlong_as_double((long long)(e + 1023) << 52);
  return ldexp(1.0, e);
}

// C of the digit split: 0x80 in each of the S - 1 lower bytes
__host__ __device__ __forceinline__ unsigned long long oz_bias(int S) {
  return 0x0080808080808080ull >> (8 * (8 - S));
}

// X + C for x 2^(8S - 2 - e), |x| < 2^e (exact scaling, round to nearest)
__device__ __forceinline__ unsigned long long oz_biased(double x, double sc, unsigned long long bias) {
  return (unsigned long long)__double2ll_rn(x * sc) + bias;
}

// digits of x (|x| < 2^e): S balanced base-256 digits, most significant first
__device__ __forceinline__ void oz_digits(double x, int e, int S, int8_t* d) {
  const double sc = e > -1000 ? pow2i(8 * S - 2 - e) : 0.0;
  const unsigned long long Y = oz_biased(x, sc, oz_bias(S));
#pragma unroll
  for (int s = 0; s < OZ_MAXS; ++s)
    if (s < S) {
      const int j = S - 1 - s;  // byte of Y
      const uint32_t b = (uint32_t)(Y >> (8 * j)) & 0xFFu;
      d[s] = (int8_t)(j == S - 1 ? b : b ^ 0x80u);
    }
}

__device__ __forceinline__ int oz_exponent(double maxabs) {
  if (!(maxabs > 0.0)) return -1000;
  int e;
  frexp(maxabs, &e);
  return e;
}


// ---- table digits, once at set-up --------------------------------------------------------
struct OzTabArgs {
  const double* leg; int H, Th2, S, NM;
  const OzProb* probs;
  const int* kidx;
  const int* nhlist;
  int8_t* B; int* fexp;
  int tab1[OZ_NTYPE], tab2[OZ_NTYPE];  // per type: table of segment 1 / segment 2
};

// Synthesis: B(column = theta row j, K = harmonic k), column scale per j.
__global__ void k_oz_tab_synth(OzTabArgs a, int type) {
  const int c = blockIdx.x, p = blockIdx.y;
  const OzProb pr = a.probs[(type * a.NM + c) * 2 + p];
  const int NC = oz_nc(type, a.S);
  for (int j = threadIdx.x; j < pr.nchunk * NC; j += blockDim.x) {
    const bool valid = j < a.Th2;
    double mx = 0.0;
    if (valid)
      for (int k = 0; k < pr.K; ++k) {
        const int t = k < pr.len1 ? a.tab1[type] : a.tab2[type];
        mx = fmax(mx, fabs(a.leg[((size_t)t * a.H + a.kidx[pr.kofs + k]) * a.Th2 + j]));
      }
    const int e = oz_exponent(mx);
    a.fexp[pr.fofs + j] = e;
    const int ch = j / NC, r = j % NC;
    for (int k = 0; k < pr.nks * 32; ++k) {
      int8_t d[OZ_MAXS];
      double v = 0.0;
      if (valid && k < pr.K) {
        const int t = k < pr.len1 ? a.tab1[type] : a.tab2[type];
        v = a.leg[((size_t)t * a.H + a.kidx[pr.kofs + k]) * a.Th2 + j];
      }
      oz_digits(v, e, a.S, d);
      for (int s = 0; s < a.S; ++s)
        a.B[pr.bofs + (((size_t)ch * pr.nks + k / 32) * a.S + s) * (NC * 32) + umma::tile_off(r, k % 32)] = d[s];
    }
  }
}

// Analysis: B(column = harmonic k of (c, p), K = folded theta row jj), column scale per k.
__global__ void k_oz_tab_anal(OzTabArgs a, int type) {
  const int c = blockIdx.x, p = blockIdx.y;
  const OzProb pr = a.probs[(type * a.NM + c) * 2 + p];
  const int NC = oz_nc(type, a.S);
  for (int k = threadIdx.x; k < pr.nchunk * NC; k += blockDim.x) {
    const bool valid = k < pr.nk;
    const int nh = valid ? a.nhlist[pr.nhofs + k] : 0;
    double mx = 0.0;
    if (valid)
      for (int jj = 0; jj < pr.K; ++jj) {
        const int t = jj < pr.len1 ? a.tab1[type] : a.tab2[type];
        const int j = jj < pr.len1 ? jj : jj - pr.len1;
        mx = fmax(mx, fabs(a.leg[((size_t)t * a.H + nh) * a.Th2 + j]));
      }
    const int e = oz_exponent(mx);
    a.fexp[pr.fofs + k] = e;
    const int cb = k / NC, r = k % NC;
    for (int jj = 0; jj < pr.nks * 32; ++jj) {
      int8_t d[OZ_MAXS];
      double v = 0.0;
      if (valid && jj < pr.K) {
        const int t = jj < pr.len1 ? a.tab1[type] : a.tab2[type];
        const int j = jj < pr.len1 ? jj : jj - pr.len1;
        v = a.leg[((size_t)t * a.H + nh) * a.Th2 + j];
      }
      oz_digits(v, e, a.S, d);
      for (int s = 0; s < a.S; ++s)
        a.B[pr.bofs + (((size_t)cb * pr.nks + jj / 32) * a.S + s) * (NC * 32) + umma::tile_off(r, jj % 32)] = d[s];
    }
  }
}

// 4 x 4 byte transpose: w[j] = byte j of x[0], x[1], x[2], x[3] (in that byte order)
__device__ __forceinline__ void byte_transpose4(const uint32_t* x, uint32_t* w) {
  const uint32_t a = __byte_perm(x[0], x[1], 0x5140), b = __byte_perm(x[0], x[1], 0x7362);
  const uint32_t c = __byte_perm(x[2], x[3], 0x5140), d = __byte_perm(x[2], x[3], 0x7362);
  w[0] = __byte_perm(a, c, 0x5410);
  w[1] = __byte_perm(a, c, 0x7632);
  w[2] = __byte_perm(b, d, 0x5410);
  w[3] = __byte_perm(b, d, 0x7632);
}

// ---- the slicing pre-pass ---------------------------------------------------------------
struct OzPrepArgs {
  int N, H, NM, Th2, HB, S, nrows, rows_per_group;
  const OzProb* probs; const int* kidx; const int* mstart; const int* mlen;
  const double* rinv;
  int8_t* A; int* erow;                  // erow [c][nrows]
  int* err;
  const cplx* in0[OZ_MAXG]; const cplx* in1[OZ_MAXG];
};

template <int TYPE> struct OzT {
  static constexpr bool anal = TYPE >= OZ_ST;
  static constexpr int per = (TYPE == OZ_P || TYPE == OZ_Q) ? 2 : 4;  // rows per shell
  static constexpr int nin = (TYPE == OZ_VEC || TYPE == OZ_ST) ? 2 : 1;
};

// One CTA = (counter c, z-block of 128 rows), both parities, in four quarters of 32 rows.
// The input rows of a quarter (the counter's harmonic segment of a shell for the
// synthesis, the (h, E/O) row of (c, n) for the analysis: contiguous in HBM) arrive by
// bulk copies (cp.async.bulk, no multicast) into one of two shared-memory stages, the
// next quarter's while this one is converted; every input value is fetched from HBM once,
// although the parity problems, K segments and row components read it up to eight times.
// Stage rows are padded to an odd number of 16-byte units, so that the shells a warp
// reads fall in distinct banks.  Every mbarrier wait is bounded; on a timeout the CTA sets
// the error flag, waits (bounded) for its copies in flight and returns.
template <int TYPE> struct OzStage {
  static constexpr int NIN = OzT<TYPE>::nin, PER = OzT<TYPE>::per, NSQ = 32 / PER;  // shells per quarter
};
template <int TYPE>
__host__ __device__ __forceinline__ size_t oz_prep_smem(int srow) {
  return sizeof(double2) * (size_t)2 * OzStage<TYPE>::NSQ * OzStage<TYPE>::NIN * srow;
}

template <int TYPE, int S>
__global__ void __launch_bounds__(256, 2) k_oz_prep(OzPrepArgs a, int srow) {
  constexpr int PER = OzT<TYPE>::per, NIN = OzT<TYPE>::nin, NSQ = OzStage<TYPE>::NSQ;
  extern __shared__ __align__(16) double2 stg[];  // [2 stages][slot][field][srow]
  __shared__ __align__(8) uint64_t full[2];
  __shared__ int e_slot[NSQ];
  __shared__ __align__(16) int kx[2][512];  // harmonic lists of the two problems (synthesis), local
                                            // indices, 0 beyond K up to the last K step
  const int c = blockIdx.x, zb = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int kbeg = a.mstart[c], klen = a.mlen[c];
  const int rowlen = OzT<TYPE>::anal ? 2 * a.Th2 : klen;  // values per (shell, field)
  const size_t stage_elems = (size_t)NSQ * NIN * srow;
  if (tid == 0) {
    umma::mbar_init(&full[0], 1);
    umma::mbar_init(&full[1], 1);
    umma::fence_mbar_init();
  }
  if (!OzT<TYPE>::anal)
    for (int p = 0; p < 2; ++p) {
      const OzProb pr = a.probs[(TYPE * a.NM + c) * 2 + p];
      for (int i = tid; i < pr.nks * 32 && i < 512; i += 256) kx[p][i] = i < pr.K ? a.kidx[pr.kofs + i] - kbeg : 0;
    }
  __syncthreads();
  // quarter q -> stage q & 1 (issued by thread 0)
  auto issue = [&](int q) {
    uint64_t* bar = &full[q & 1];
    double2* dst = stg + (size_t)(q & 1) * stage_elems;
    const int R0 = zb * 128 + q * 32;
    uint32_t bytes = 0;
    for (int sl = 0; sl < NSQ; ++sl)
      if (R0 + sl * PER < a.nrows) bytes += NIN * rowlen * 16;
    umma::mbar_expect_tx(bar, bytes);
    for (int sl = 0; sl < NSQ; ++sl) {
      const int R = R0 + sl * PER;
      if (R >= a.nrows) break;
      const int g = R / a.rows_per_group, n = (R % a.rows_per_group) / PER;
      for (int f = 0; f < NIN; ++f) {
        const cplx* src = f == 0 ? a.in0[g] : a.in1[g];
        src += OzT<TYPE>::anal ? four_off_a(n, c, 0, 0, a.N, a.Th2) : (size_t)n * a.H + kbeg;
        umma::bulk_g2s(dst + (size_t)(sl * NIN + f) * srow, src, (uint32_t)rowlen * 16, bar);
      }
    }
  };
  if (tid == 0) { issue(0); issue(1); }
  // thread = (row r of the quarter, warp kq): the synthesis gives warp kq the K eighth kq of
  // every K step, the analysis whole (K step, 16-byte half) items in turn (below)
  const int r = tid & 31, kq = tid >> 5;
  for (int q = 0; q < 4; ++q) {
    const int R0 = zb * 128 + q * 32;
    const double2* st = stg + (size_t)(q & 1) * stage_elems;
    const bool got = umma::mbar_wait(&full[q & 1], (q >> 1) & 1, WAIT_ITERS);
    if (__syncthreads_or(!got)) {  // give up: flag, let the copies in flight land, leave
      if (tid == 0) {
        atomicExch(a.err, 1);
        for (int qq = q; qq < 4 && qq < q + 2; ++qq) umma::mbar_wait(&full[qq & 1], (qq >> 1) & 1, WAIT_ITERS);
      }
      __syncthreads();
      return;
    }
    // ---- exponents: one warp per shell, max over the staged values of its fields
    for (int sl = warp; sl < NSQ; sl += 8) {
      const int R = R0 + sl * PER;
      const double r1 = (TYPE == OZ_GRAD && R < a.nrows) ? a.rinv[(R % a.rows_per_group) / PER] : 1.0;
      double mx = 0.0;
      if (R < a.nrows)
        for (int i = lane; i < NIN * rowlen; i += 32) {
          const int f = i / rowlen, k = i - f * rowlen;
          double2 v = st[(size_t)(sl * NIN + f) * srow + k];
          if (TYPE == OZ_GRAD) { v.x *= r1; v.y *= r1; }
          mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
        }
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0) e_slot[sl] = oz_exponent(mx);
    }
    __syncthreads();
    if (tid < 32 && R0 + tid < a.nrows) a.erow[(size_t)c * a.nrows + R0 + tid] = e_slot[tid / PER];
    // ---- digits of both parities' A tiles: the bytes of X + C (oz_digits) of four values
    // make one 32-bit word per slice (a byte transpose of their low and high words), bit 7
    // flipped in all but the top slice.
    const int R = R0 + r;
    const bool live = R < a.nrows;
    const int sl = r / PER, comp = R % PER;
    const double sc = live && e_slot[sl] > -1000 ? pow2i(8 * S - 2 - e_slot[sl]) : 0.0;
    const unsigned long long bias = oz_bias(S);
    const double* row0 = (const double*)(st + (size_t)(sl * NIN) * srow);
    const double* row1 = row0 + 2 * srow;  // second field (VEC: t, ST: phi)
    const int rt = q * 32 + r;             // row inside the 128-row tile
    // Per thread and K segment, the value of K slot k is f * src[idx(k)] (a double of the
    // staged complex rows: component and field fixed by the row's component `comp`), and f
    // (a sign, 1/r for the gradient, 0 where the segment does not feed this component) is
    // folded into the power-of-two scale: fl(x f 2^a) = fl(x f) 2^a, so the digits are
    // those of the value itself.  The reference's recipes:
    //  VEC theta: s llP_ (segment 1) + (t.im, -t.re) llsin1mP (segment 2);
    //      phi:   t llP_ + (-s.im, s.re) llsin1mP                      (transform.fftw3.F90:746-774)
    //  GRAD theta: (C/r) P_ ; phi: i (C/r) sin1mP                     (transform.fftw3.F90:955-1000)
    //  ST s: Yth gwllP_ + (Yph.im, -Yph.re) gwllsin1mP ; t: Yph gwllP_ + (-Yth.im, Yth.re),
    //      segment 1 on parity 1 - p, segment 2 on parity p             (transform.fftw3.F90:866-909)
    const double* src1;  // segment 1 (k < len1)
    const double* src2;  // segment 2
    double f1 = 1.0, f2 = 1.0;
    if (TYPE == OZ_P || TYPE == OZ_Q) {
      src1 = src2 = row0 + (comp & 1);
    } else if (TYPE == OZ_VEC || TYPE == OZ_ST) {
      src1 = (comp >= 2 ? row1 : row0) + (comp & 1);
      src2 = (comp < 2 ? row1 : row0) + ((comp & 1) ? 0 : 1);
      f2 = (comp == 1 || comp == 2) ? -1.0 : 1.0;
    } else {  // OZ_GRAD
      const double r1 = live ? a.rinv[(R % a.rows_per_group) / PER] : 1.0;
      src1 = row0 + (comp & 1);
      src2 = row0 + (comp == 2 ? 1 : 0);
      f1 = comp < 2 ? r1 : 0.0;
      f2 = comp >= 2 ? (comp == 2 ? -r1 : r1) : 0.0;
    }
    const double sc1 = sc * f1, sc2 = sc * f2;
    if constexpr (OzT<TYPE>::anal) {
      // items (parity, K step, 16-byte half of the step) over the warps; a thread writes one
      // full 16-byte core-matrix row per slice, a warp four whole 128-byte lines (the
      // analysis has K steps enough for all warps).  Slot k reads complex element 2j + pp
      // (j = k in segment 1, k - len1 in segment 2; pp = 1 - p, p (ST) or p (Q)), i.e. the
      // double 4k + const per segment.
      const OzProb pr0 = a.probs[(TYPE * a.NM + c) * 2], pr1 = a.probs[(TYPE * a.NM + c) * 2 + 1];
      const int n0 = pr0.nchunk ? 2 * pr0.nks : 0, n1 = pr1.nchunk ? 2 * pr1.nks : 0;
      for (int i = kq; i < n0 + n1; i += 8) {
        const int p = i < n0 ? 0 : 1;
        const OzProb& pr = p ? pr1 : pr0;
        const int li = i - (p ? n0 : 0), ks = li >> 1, hh = li & 1;
        const int pp1 = TYPE == OZ_ST ? 1 - p : p;
        const double* b1 = src1 + 2 * pp1;
        const double* b2 = src2 + 2 * p - 4 * pr.len1;
        int8_t* Ablk = a.A + pr.aofs + (size_t)zb * pr.nks * S * 4096;
        uint32_t ow[S][4];
#pragma unroll
        for (int b4 = 0; b4 < 4; ++b4) {
          uint32_t hi[4], lo[4];
#pragma unroll
          for (int u4 = 0; u4 < 4; ++u4) {
            const int k = ks * 32 + hh * 16 + b4 * 4 + u4;
            const bool s1 = k < pr.len1;
            const double x = (live && k < pr.K) ? (s1 ? b1 : b2)[4 * k] : 0.0;
            const unsigned long long Y = oz_biased(x, s1 ? sc1 : sc2, bias);
            lo[u4] = (uint32_t)Y;
            hi[u4] = (uint32_t)(Y >> 32);
          }
          uint32_t wl[4], wh[4];
          byte_transpose4(lo, wl);
          if (S > 4) byte_transpose4(hi, wh);
#pragma unroll
          for (int s2 = 0; s2 < S; ++s2) {
            const int j = S - 1 - s2;  // slice s2 = byte j of X + C
            const uint32_t w = j >= 4 ? wh[j - 4] : wl[j];
            ow[s2][b4] = j == S - 1 ? w : w ^ 0x80808080u;
          }
        }
        const int toff = umma::tile_off(rt, hh * 16);
#pragma unroll
        for (int s2 = 0; s2 < S; ++s2)
          *(uint4*)(Ablk + ((size_t)ks * S + s2) * 4096 + toff) =
              make_uint4(ow[s2][0], ow[s2][1], ow[s2][2], ow[s2][3]);
      }
    } else {
      // thread (row, K eighth kq): four values of every K step, one 32-bit word per slice
      // (the synthesis has few K steps per counter); slot k reads complex element kx[p][k]
      for (int p = 0; p < 2; ++p) {
        const OzProb pr = a.probs[(TYPE * a.NM + c) * 2 + p];
        if (pr.nchunk == 0) continue;
        int8_t* Ablk = a.A + pr.aofs + (size_t)zb * pr.nks * S * 4096;
        for (int ks = 0; ks < pr.nks; ++ks) {
          const int kb = ks * 32 + kq * 4;
          const int4 k4 = *(const int4*)&kx[p][kb];
          const int ke[4] = {k4.x, k4.y, k4.z, k4.w};
          uint32_t hi[4], lo[4];
#pragma unroll
          for (int u4 = 0; u4 < 4; ++u4) {
            const int k = kb + u4;
            const bool s1 = k < pr.len1;
            const double x = (live && k < pr.K) ? (s1 ? src1 : src2)[2 * ke[u4]] : 0.0;
            const unsigned long long Y = oz_biased(x, s1 ? sc1 : sc2, bias);
            lo[u4] = (uint32_t)Y;
            hi[u4] = (uint32_t)(Y >> 32);
          }
          uint32_t wl[4], wh[4];
          byte_transpose4(lo, wl);
          if (S > 4) byte_transpose4(hi, wh);
          const int toff = umma::tile_off(rt, kq * 4);
#pragma unroll
          for (int s2 = 0; s2 < S; ++s2) {
            const int j = S - 1 - s2;  // slice s2 = byte j of X + C
            const uint32_t w = j >= 4 ? wh[j - 4] : wl[j];
            *(uint32_t*)(Ablk + ((size_t)ks * S + s2) * 4096 + toff) = j == S - 1 ? w : w ^ 0x80808080u;
          }
        }
      }
    }
    __syncthreads();  // stage q & 1 fully read
    if (tid == 0 && q + 2 < 4) issue(q + 2);
  }
}

// ---- the GEMM ---------------------------------------------------------------------------
struct OzGemmArgs {
  int N, H, NM, Th2, HB, S, nrows, rows_per_group;
  const OzProb* probs; const int8_t* A; const int8_t* B; const int* fexp; const int* erow;
  const int* nhlist; const int* hm;
  cplx* out0[OZ_MAXG]; cplx* out1[OZ_MAXG]; int zero_m0_im[OZ_MAXG];
  int* err;
  int nst;          // stages of the bulk-copy ring
  int pair_digits;  // the launch's diagonal bound allows D_2i 256 + D_2i+1 in int32
  int wide_sum;     // ... and the whole sum over the diagonals in int64 (oz_combine)
};

// one 32-byte store of two complex values (p 32-byte aligned)
__device__ __forceinline__ void st_global_2c(cplx* p, double2 a, double2 b) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y)
               : "memory");
}

// The integer sum_d D_d 256^(S-1-d) of one accumulator column.  wide (the host's bound
// on the sum is below 2^62): formed exactly in int64 and converted once (exact while
// |sum| < 2^53, one rounding beyond); else a Horner sum in FP64 (exact below 2^53).
// pair: two diagonals per int32 first (D_2i 256 + D_2i+1, which the host has bounded
// below 2^31), then 2^16 steps: half the steps, and in FP64 half the conversions.
template <int S, int W>
__device__ __forceinline__ double oz_combine(const int32_t (&v)[S][W], int q, bool pair, bool wide) {
  if (wide) {
    long long h;
    if (pair) {
      h = (long long)(v[0][q] * 256 + v[1][q]);
#pragma unroll
      for (int d = 2; d < S; d += 2)
        if (d + 1 < S) h = h * 65536 + (long long)(v[d][q] * 256 + v[d + 1][q]);
        else h = h * 256 + (long long)v[d][q];
    } else {
      h = (long long)v[0][q];
#pragma unroll
      for (int d = 1; d < S; ++d) h = h * 256 + (long long)v[d][q];
    }
    return (double)h;
  }
  double h;
  if (pair) {
    h = (double)(v[0][q] * 256 + v[1][q]);
#pragma unroll
    for (int d = 2; d < S; d += 2)
      if (d + 1 < S) h = fma(h, 65536.0, (double)(v[d][q] * 256 + v[d + 1][q]));
      else h = fma(h, 256.0, (double)v[d][q]);
  } else {
    h = (double)v[0][q];
#pragma unroll
    for (int d = 1; d < S; ++d) h = fma(h, 256.0, (double)v[d][q]);
  }
  return h;
}

__device__ __forceinline__ bool oz_wait(uint64_t* mbar, uint32_t parity, int* err) {
  if (umma::mbar_wait(mbar, parity, WAIT_ITERS)) return true;
  atomicExch(err, 1);
  return false;
}

// Persistent: CTA b walks the tiles t = b, b + gridDim.x, ... of the (counter c, parity p,
// z-block of 128 rows) grid, each a loop over column chunks.  The bulk-copy ring, the MMA
// issue and the tensor-memory handshakes run on counters over all of the CTA's tiles, so
// the pipeline does not drain between tiles.  Two CTAs per SM (256 tensor-memory columns
// each).
template <int TYPE, int S>
__global__ void __launch_bounds__(OZ_THREADS, 2) k_oz_gemm(OzGemmArgs a, int nzb) {
  constexpr int PER = OzT<TYPE>::per;
  extern __shared__ __align__(1024) uint8_t oz_smem[];
  __shared__ __align__(8) uint64_t full[OZ_MAXSTAGES], empty[OZ_MAXSTAGES], accf, tfree, fin;
  __shared__ uint32_t tbase;
  __shared__ double csc[2][OZ_NCMAX];  // column scales 2^fexp of a chunk (chunk parity)
  constexpr int NC = oz_nc(TYPE, S), BT = NC * 32;  // chunk columns; bytes of one B slice tile
  const int tid = threadIdx.x, warp = tid >> 5;
  const int ntile = a.NM * 2 * nzb;
  const uint32_t stage_bytes = (uint32_t)S * (4096 + BT);  // A: S x 4096, B: S x BT
  const int nst = a.nst;
  if (tid == 0) {
    for (int i = 0; i < nst; ++i) { umma::mbar_init(&full[i], 1); umma::mbar_init(&empty[i], 1); }
    umma::mbar_init(&accf, 1);
    umma::mbar_init(&tfree, OZ_EPI);
    umma::mbar_init(&fin, 1);
    umma::fence_mbar_init();
  }
  if (warp == 0) umma::tmem_alloc(&tbase, 256);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tbase;
  // tile t -> (c, p, zb), z-block fastest
  auto tile = [&](int t, int& c, int& p, int& zb) {
    zb = t % nzb;
    p = (t / nzb) & 1;
    c = t / (2 * nzb);
  };
  // the problem of tile t (loaded one tile ahead, so the load's latency is hidden)
  auto prob = [&](int t) {
    OzProb pr{};
    if (t < ntile) {
      int c, p, zb;
      tile(t, c, p, zb);
      pr = a.probs[(TYPE * a.NM + c) * 2 + p];
    }
    return pr;
  };

  if (tid == OZ_EPI) {
    // ---- producer: A (z-block, K step) and B (chunk, K step) tiles into the ring
    int it = 0;
    bool ok = true;
    OzProb nxt = prob(blockIdx.x);
    for (int t = blockIdx.x; t < ntile && ok; t += gridDim.x) {
      int c, p, zb;
      tile(t, c, p, zb);
      const OzProb pr = nxt;
      nxt = prob(t + gridDim.x);
      const int8_t* Ablk = a.A + pr.aofs + (size_t)zb * pr.nks * S * 4096;
      const int8_t* Bblk = a.B + pr.bofs;
      for (int q = 0; q < pr.nchunk * pr.nks; ++q, ++it) {
        const int st = it % nst, use = it / nst;
        if (use > 0 && !oz_wait(&empty[st], (use - 1) & 1, a.err)) { ok = false; break; }
        const int ch = q / pr.nks, ks = q % pr.nks;
        uint8_t* sA = oz_smem + (size_t)st * stage_bytes;
        umma::mbar_expect_tx(&full[st], stage_bytes);
        umma::bulk_g2s(sA, Ablk + (size_t)ks * S * 4096, (uint32_t)S * 4096, &full[st]);
        umma::bulk_g2s(sA + (size_t)S * 4096, Bblk + ((size_t)ch * pr.nks + ks) * S * BT, (uint32_t)S * BT,
                       &full[st]);
      }
    }
    // drain: the copies of the last stages have landed before the CTA can exit
    for (int j = (it > nst ? it - nst : 0); j < it; ++j)
      umma::mbar_wait(&full[j % nst], (j / nst) & 1, WAIT_ITERS);
  } else if (tid == OZ_EPI + 32) {
    // ---- MMA issuer: the S(S+1)/2 digit pairs of a K step into S diagonals of NC columns,
    // as S MMAs: A slice sa against B slices 0 .. S-1-sa at once (stacked in the stage, they
    // are one K-major operand of N = NC (S - sa) rows), accumulating into the tensor-memory
    // columns NC sa .. NC S - 1, i.e. diagonals d = sa + s
    int it = 0, cc = 0;
    bool ok = true;
    OzProb nxt = prob(blockIdx.x);
    for (int t = blockIdx.x; t < ntile && ok; t += gridDim.x) {
      const OzProb pr = nxt;
      nxt = prob(t + gridDim.x);
      for (int ch = 0; ch < pr.nchunk && ok; ++ch, ++cc) {
        if (cc > 0 && !oz_wait(&tfree, (cc - 1) & 1, a.err)) { ok = false; break; }
        umma::fence_after_sync();
        for (int ks = 0; ks < pr.nks; ++ks, ++it) {
          const int st = it % nst;
          if (!oz_wait(&full[st], (it / nst) & 1, a.err)) { ok = false; break; }
          umma::fence_after_sync();
          const uint32_t sa0 = umma::smem_u32(oz_smem + (size_t)st * stage_bytes);
          const uint32_t sb0 = sa0 + (uint32_t)S * 4096;
          const uint64_t bd = umma::desc_kmajor_noswz(sb0, 128, 256);
          for (int sa = 0; sa < S; ++sa) {
            const uint64_t ad = umma::desc_kmajor_noswz(sa0 + (uint32_t)sa * 4096, 128, 256);
            umma::mma_s8(tmem + (uint32_t)(sa * NC), ad, bd, umma::idesc_s8(128, NC * (S - sa)),
                         (ks > 0 || sa > 0) ? 1 : 0);
          }
          umma::commit(&empty[st]);
        }
        if (ok) umma::commit(&accf);
      }
    }
    umma::commit(&fin);  // arrives when every MMA issued above has completed
    umma::mbar_wait(&fin, 0, WAIT_ITERS);
  } else if (tid < OZ_EPI) {
    // ---- epilogue: row (tid mod 128) of each z-block, the half tid / 128 of a chunk's NC
    // columns, in groups of CW.  Per group the thread reads its S x CW accumulator words,
    // forms the CW values, trades half of them with the neighbouring lane (rows 2i and
    // 2i + 1 are Re and Im of one output: the even lane keeps the group's first CW/2
    // columns, the odd lane the rest) and stores its complex values straight to HBM.  The
    // tensor memory goes back once the last group's words are in registers (the MMAs of
    // the next chunk run while the thread converts and stores).
    const int row = tid & 127, half = tid >> 7, odd = row & 1;
    const uint32_t tlane = (uint32_t)(32 * (warp & 3)) << 16;
    const bool pair = a.pair_digits != 0, wide = a.wide_sum != 0;
    int cc = 0;
    OzProb nxt = prob(blockIdx.x);
    for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
      int c, p, zb;
      tile(t, c, p, zb);
      const OzProb pr = nxt;
      nxt = prob(t + gridDim.x);
      if (pr.nchunk == 0) continue;  // no harmonics of this parity: nothing to write
      const int R = zb * 128 + row, Rp = R & ~1;  // rows come in (Re, Im) pairs: nrows is even
      const bool live = R < a.nrows;
      cplx* base = nullptr;  // this lane pair's output
      bool zero = false;     // analysis: drop the imaginary part of m = 0
      if (Rp < a.nrows) {
        const int g = Rp / a.rows_per_group, n = (Rp % a.rows_per_group) / PER, comp = Rp % PER;
        cplx* out = (comp < 2) ? a.out0[g] : a.out1[g];
        base = OzT<TYPE>::anal ? out + (size_t)n * a.H : out + four_off(n, c, p, 0, a.NM, a.HB);
        zero = TYPE == OZ_ST || a.zero_m0_im[g];
      }
      // x y = 2^(ea + eb + 4) sum_d D_d 2^(-8(d+2)) = 2^(ea + eb + 4 - 8(S+1)) H with
      // H = Horner over d in 2^8; the power of two and the row scale 2^erow are one factor
      const double rsc = live ? pow2i(a.erow[(size_t)c * a.nrows + R] + 4 - 8 * (S + 1)) : 0.0;
      bool ok = true;
      for (int ch = 0; ch < pr.nchunk; ++ch, ++cc) {
        // csc[cc & 1] was last read in chunk cc - 2, before every thread's barrier of cc - 1
        if (tid < NC) csc[cc & 1][tid] = pow2i(a.fexp[pr.fofs + ch * NC + tid]);
        const bool got = umma::mbar_wait(&accf, cc & 1, WAIT_ITERS);
        if (!umma::bar_and(1, OZ_EPI, got)) {  // uniform over the epilogue threads
          if (tid == 0) atomicExch(a.err, 1);
          ok = false;
          break;
        }
        umma::fence_after_sync();
        constexpr int NH = NC / 2;  // columns of a thread's half of the chunk
        const double* cs = csc[cc & 1] + NH * half;
        // groups of CW columns (8 up to five slices, 4 above, to bound the registers); per
        // group the even lane keeps its first HW columns, the odd lane the last HW
        constexpr int CW = S <= 5 ? 8 : 4, NGR = NH / CW, HW = CW / 2;
#pragma unroll
        for (int gi = 0; gi < NGR; ++gi) {
          int32_t v[S][CW];
#pragma unroll
          for (int d = 0; d < S; ++d) {
            const uint32_t ta = tmem + tlane + (uint32_t)(d * NC + NH * half + CW * gi);
            if constexpr (CW == 8) umma::tmem_ld8(ta, v[d]);
            else umma::tmem_ld4(ta, v[d]);
          }
          umma::tmem_wait_ld();
          if (gi == NGR - 1) {  // all words of this chunk are in registers
            umma::fence_before_sync();
            umma::mbar_arrive(&tfree);
          }
          double h[CW];
#pragma unroll
          for (int q = 0; q < CW; ++q) h[q] = oz_combine<S, CW>(v, q, pair, wide) * (rsc * cs[CW * gi + q]);
          double2 o[HW];
#pragma unroll
          for (int q = 0; q < HW; ++q) {
            const double r = __shfl_xor_sync(0xffffffffu, odd ? h[q] : h[q + HW], 1);
            o[q] = odd ? make_double2(r, h[q + HW]) : make_double2(h[q], r);
          }
          if (base) {  // stored group by group (fewer live registers)
            const int k0 = ch * NC + NH * half + CW * gi + HW * odd;
            if (!OzT<TYPE>::anal) {
              // theta rows j, j + 1 (j even) of one half-row pair are neighbours in four_off:
              // one 32-byte store (the field bases are 32-byte aligned)
#pragma unroll
              for (int q = 0; q < HW; q += 2) {
                const int j = k0 + q;
                cplx* dst = base + (size_t)(j >> 1) * a.NM * 4;
                if (j + 1 < a.Th2) st_global_2c(dst, o[q], o[q + 1]);
                else if (j < a.Th2) *dst = o[q];
              }
            } else {
#pragma unroll
              for (int q = 0; q < HW; ++q) {
                const int k = k0 + q;
                if (k < pr.nk) {
                  const int nh = a.nhlist[pr.nhofs + k];
                  double2 val = o[q];
                  // m = 0: s, t (and a scalar) keep no imaginary part; q keeps its own
                  // (transform.fftw3.F90:599, 869, 902, 908)
                  if (zero && a.hm[nh] == 0) val.y = 0.0;
                  base[nh] = val;
                }
              }
            }
          }
        }
      }
      if (!ok) break;
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 256);
}

}  // namespace

// =========================================================================================
// host side
// =========================================================================================
struct OzState {
  int S = 0;
  int nzb_max[OZ_NTYPE] = {};
  OzProb* d_probs = nullptr;
  int* d_kidx = nullptr;
  int* d_nh = nullptr;
  int8_t* d_B = nullptr;
  int* d_fexp = nullptr;
  // data digits and row exponents [c][rows], one buffer per concurrent chain: synthesis
  // VEC / P / GRAD and analysis ST / Q run as forked branches (buffer 0: VEC, ST; 1: P, Q;
  // 2: GRAD), the two phases never at once
  int8_t* d_A[3] = {};
  int* d_erow[3] = {};
  // per stream that launches a contraction (the context's stream, or a graph-capture
  // stream): two more streams and the fork / join events of its branches.  A stream that
  // joined one capture stays in it until that capture ends, so nested captures need
  // streams of their own.
  struct Aux { cudaStream_t origin; cudaStream_t s[2]; cudaEvent_t fork, join[2]; };
  std::vector<Aux> aux;
  int* d_err = nullptr;
  size_t smem = 0;
  int nst = 2;           // GEMM ring stages
  int ctas = 2;          // persistent GEMM CTAs per SM
  int srow[2] = {1, 1};  // pre-pass stage row length (odd, in complex): synthesis, analysis
  int pair[OZ_NTYPE] = {};  // per type: the epilogue may join diagonals in pairs (oz_combine)
  int wide[OZ_NTYPE] = {};  // per type: ... and sum them in int64
};

namespace {
constexpr int OZ_MAXG_SYNTH = OZ_MAXG, OZ_MAXG_ANAL = 4;  // groups per launch

// the digit / exponent buffer of each type's chain
int oz_buf(int type) { return type == OZ_VEC || type == OZ_ST ? 0 : type == OZ_P || type == OZ_Q ? 1 : 2; }

// f(k_oz_gemm<TYPE, S>) for the runtime slice count S
template <int TYPE, class F>
void oz_gemm_dispatch(int S, F&& f) {
  switch (S) {
    case 2: f(k_oz_gemm<TYPE, 2>); break;
    case 3: f(k_oz_gemm<TYPE, 3>); break;
    case 4: f(k_oz_gemm<TYPE, 4>); break;
    case 5: f(k_oz_gemm<TYPE, 5>); break;
    case 6: f(k_oz_gemm<TYPE, 6>); break;
    case 7: f(k_oz_gemm<TYPE, 7>); break;
    default: f(k_oz_gemm<TYPE, 8>); break;
  }
}
template <int TYPE>
void oz_set_smem(int S, size_t smem) {
  oz_gemm_dispatch<TYPE>(S, [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
}
}  // namespace

void lsd_ozaki_free(lsd_ctx* ctx) {
  OzState* o = (OzState*)ctx->oz;
  if (!o) return;
  void* ptrs[] = {o->d_probs, o->d_kidx, o->d_nh, o->d_B, o->d_fexp, o->d_A[0], o->d_A[1], o->d_A[2],
                  o->d_erow[0], o->d_erow[1], o->d_erow[2], o->d_err};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  for (OzState::Aux& x : o->aux) {
    for (int i = 0; i < 2; ++i) {
      if (x.s[i]) cudaStreamDestroy(x.s[i]);
      if (x.join[i]) cudaEventDestroy(x.join[i]);
    }
    if (x.fork) cudaEventDestroy(x.fork);
  }
  delete o;
  ctx->oz = nullptr;
}

int lsd_ozaki_setup(lsd_ctx* ctx) {
  OzState* o = new OzState();
  ctx->oz = o;
  const int S = ctx->cfg.ozaki_slices > 0 ? ctx->cfg.ozaki_slices : 7;
  if (S < 2 || S > OZ_MAXS) return lsd_fail(ctx, LSD_EARG, "ozaki_slices must be 2..8");
  o->S = S;
  const int NM = ctx->NM, Th2 = ctx->Th2, N = ctx->N;
  for (int c = 0; c < NM; ++c)
    if (ctx->mlen[c] > 512) return lsd_fail(ctx, LSD_EARG, "tensor-core path: more than 512 harmonics per m");
  std::vector<std::vector<int>> Kcp((size_t)NM * 2);  // harmonics per (counter, parity)
  for (int c = 0; c < NM; ++c)
    for (int k = 0; k < ctx->mlen[c]; ++k) {
      const int nh = ctx->mstart[c] + k;
      Kcp[(size_t)c * 2 + ctx->hs[nh]].push_back(nh);
    }
  std::vector<int> kidx, nhl;
  std::vector<OzProb> probs((size_t)OZ_NTYPE * NM * 2);
  long long bbytes = 0, abytes_t[OZ_NTYPE] = {};
  int fofs = 0;
  for (int type = 0; type < OZ_NTYPE; ++type) {
    const bool anal = type >= OZ_ST;
    const int per = (type == OZ_P || type == OZ_Q) ? 2 : 4;
    const int maxg = anal ? OZ_MAXG_ANAL : OZ_MAXG_SYNTH;
    o->nzb_max[type] = ceil_div(maxg * per * N, 128);
    long long abytes = 0;
    for (int c = 0; c < NM; ++c)
      for (int p = 0; p < 2; ++p) {
        OzProb pr{};
        const std::vector<int>& Kp = Kcp[(size_t)c * 2 + p];
        const std::vector<int>& Kq = Kcp[(size_t)c * 2 + 1 - p];
        pr.nhofs = (int)nhl.size();
        pr.nk = (int)Kp.size();
        nhl.insert(nhl.end(), Kp.begin(), Kp.end());
        pr.kofs = (int)kidx.size();
        if (type == OZ_VEC || type == OZ_GRAD) {
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
        // analysis: (c, p) without harmonics has no output (nchunk 0); a synthesis output
        // without harmonics is still written (zeros)
        const bool empty = anal && pr.nk == 0;
        const int NC = oz_nc(type, S);
        pr.nchunk = empty ? 0 : (anal ? ceil_div(pr.nk, NC) : ceil_div(Th2, NC));
        pr.fofs = fofs;
        fofs += pr.nchunk * NC;
        pr.bofs = bbytes;
        bbytes += (long long)pr.nchunk * pr.nks * S * NC * 32;
        pr.aofs = abytes;
        if (pr.nchunk) abytes += (long long)o->nzb_max[type] * pr.nks * S * 4096;
        probs[((size_t)type * NM + c) * 2 + p] = pr;
      }
    abytes_t[type] = abytes;
    // digit products bound the diagonals: |D_d| <= K sum_{s+t=d} m_s m_t with m_0 = 65 (the
    // top digit) and m_s = 128 below it; pairs need 256 |D_2i| + |D_2i+1| < 2^31
    long long kmax = 0;
    for (int c = 0; c < NM; ++c)
      for (int p = 0; p < 2; ++p) kmax = std::max(kmax, 32LL * probs[((size_t)type * NM + c) * 2 + p].nks);
    auto bound = [&](int d) {
      long long b = 0;
      for (int s = 0; s < S; ++s) {
        const int t = d - s;
        if (t >= 0 && t < S) b += (long long)(s ? 128 : 65) * (t ? 128 : 65);
      }
      return kmax * b;
    };
    bool pair_ok = true;
    for (int d = 0; d + 1 < S; d += 2) pair_ok = pair_ok && 256 * bound(d) + bound(d + 1) < (1LL << 31);
    o->pair[type] = pair_ok ? 1 : 0;
    double total = 0.0;  // bound on |sum_d D_d 256^(S-1-d)|
    for (int d = 0; d < S; ++d) total += (double)bound(d) * std::ldexp(1.0, 8 * (S - 1 - d));
    o->wide[type] = total < std::ldexp(1.0, 62) ? 1 : 0;
  }
  // ring stages: as many (2..4) as keep two CTAs per SM (<= 78 KiB of stages each)
  lsd_ozaki_default_tiles(S, &o->nst, &o->ctas);
  o->smem = (size_t)o->nst * oz_stage_bytes(S);
  {
    int mx = 1;
    for (int c = 0; c < NM; ++c) mx = std::max(mx, ctx->mlen[c]);
    o->srow[0] = mx | 1;
    o->srow[1] = (2 * Th2) | 1;
    if (oz_prep_smem<OZ_ST>(o->srow[1]) > 200 * 1024 || oz_prep_smem<OZ_VEC>(o->srow[0]) > 200 * 1024)
      return lsd_fail(ctx, LSD_EARG, "tensor-core path: pre-pass rows do not fit in shared memory");
  }
  if (kidx.empty()) kidx.push_back(0);
  if (nhl.empty()) nhl.push_back(0);
  CUDA_TRY(cudaMalloc(&o->d_probs, sizeof(OzProb) * probs.size()));
  // uploads on the context's stream, which the table kernels below run on
  CUDA_TRY(cudaMemcpyAsync(o->d_probs, probs.data(), sizeof(OzProb) * probs.size(), cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaMalloc(&o->d_kidx, sizeof(int) * kidx.size()));
  CUDA_TRY(cudaMemcpyAsync(o->d_kidx, kidx.data(), sizeof(int) * kidx.size(), cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaMalloc(&o->d_nh, sizeof(int) * nhl.size()));
  CUDA_TRY(cudaMemcpyAsync(o->d_nh, nhl.data(), sizeof(int) * nhl.size(), cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaMalloc(&o->d_B, std::max<long long>(bbytes, 16)));
  CUDA_TRY(cudaMalloc(&o->d_fexp, sizeof(int) * (size_t)std::max(fofs, 1)));
  for (int b = 0; b < 3; ++b) {  // the buffers of the chains (oz_buf)
    long long ab = 16;
    int rows = 128;
    for (int type = 0; type < OZ_NTYPE; ++type)
      if (oz_buf(type) == b) {
        ab = std::max(ab, abytes_t[type]);
        rows = std::max(rows, o->nzb_max[type] * 128);
      }
    CUDA_TRY(cudaMalloc(&o->d_A[b], ab));
    CUDA_TRY(cudaMalloc(&o->d_erow[b], sizeof(int) * (size_t)NM * rows));
  }
  CUDA_TRY(cudaMalloc(&o->d_err, sizeof(int)));
  CUDA_TRY(cudaMemsetAsync(o->d_err, 0, sizeof(int), ctx->stream));
  OzTabArgs ta;
  ta.leg = ctx->d_leg; ta.H = ctx->H; ta.Th2 = Th2; ta.S = S; ta.NM = NM;
  ta.probs = o->d_probs; ta.kidx = o->d_kidx; ta.nhlist = o->d_nh; ta.B = o->d_B; ta.fexp = o->d_fexp;
  const int t1[OZ_NTYPE] = {LSD_LEG_LLP_, LSD_LEG_P, LSD_LEG_P_, LSD_LEG_GWLLP_, LSD_LEG_GWP};
  const int t2[OZ_NTYPE] = {LSD_LEG_LLSIN1MP, LSD_LEG_P, LSD_LEG_SIN1MP, LSD_LEG_GWLLSIN1MP, LSD_LEG_GWP};
  for (int i = 0; i < OZ_NTYPE; ++i) { ta.tab1[i] = t1[i]; ta.tab2[i] = t2[i]; }
  const dim3 g(NM, 2);
  for (int type = OZ_VEC; type <= OZ_GRAD; ++type) k_oz_tab_synth<<<g, 128, 0, ctx->stream>>>(ta, type);
  for (int type = OZ_ST; type <= OZ_Q; ++type) k_oz_tab_anal<<<g, 64, 0, ctx->stream>>>(ta, type);
  ctx->launches += 5;
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  oz_set_smem<OZ_VEC>(o->S, o->smem); oz_set_smem<OZ_P>(o->S, o->smem); oz_set_smem<OZ_GRAD>(o->S, o->smem);
  oz_set_smem<OZ_ST>(o->S, o->smem); oz_set_smem<OZ_Q>(o->S, o->smem);
  CUDA_TRY(cudaGetLastError());
  return LSD_OK;
}

namespace {

struct OzLaunchGroup { const cplx* in0; const cplx* in1; cplx* out0; cplx* out1; int zero_m0_im; };

template <int TYPE>
int oz_run(lsd_ctx* ctx, const OzLaunchGroup* gs, int ng, cudaStream_t stream) {
  OzState* o = (OzState*)ctx->oz;
  const int buf = oz_buf(TYPE);
  constexpr int PER = OzT<TYPE>::per;
  const int rpg = PER * ctx->N, nrows = ng * rpg, nzb = ceil_div(nrows, 128);
  if (nzb > o->nzb_max[TYPE]) return lsd_fail(ctx, LSD_EARG, "tensor-core contraction: too many groups in one launch");
  OzPrepArgs pa;
  pa.N = ctx->N; pa.H = ctx->H; pa.NM = ctx->NM; pa.Th2 = ctx->Th2; pa.HB = ctx->HB; pa.S = o->S; pa.nrows = nrows;
  pa.rows_per_group = rpg; pa.probs = o->d_probs; pa.kidx = o->d_kidx; pa.mstart = ctx->d_mstart;
  pa.mlen = ctx->d_mlen; pa.rinv = ctx->d_rinv; pa.A = o->d_A[buf]; pa.erow = o->d_erow[buf];
  pa.err = o->d_err;
  OzGemmArgs ga;
  ga.N = ctx->N; ga.H = ctx->H; ga.NM = ctx->NM; ga.Th2 = ctx->Th2; ga.HB = ctx->HB; ga.S = o->S; ga.nrows = nrows;
  ga.rows_per_group = rpg; ga.probs = o->d_probs; ga.A = o->d_A[buf]; ga.B = o->d_B; ga.fexp = o->d_fexp;
  ga.erow = o->d_erow[buf]; ga.nhlist = o->d_nh; ga.hm = ctx->d_m; ga.err = o->d_err; ga.nst = o->nst;
  ga.pair_digits = o->pair[TYPE];
  ga.wide_sum = o->wide[TYPE];
  for (int i = 0; i < OZ_MAXG; ++i) {
    const bool on = i < ng;
    pa.in0[i] = on ? gs[i].in0 : nullptr; pa.in1[i] = on ? gs[i].in1 : nullptr;
    ga.out0[i] = on ? gs[i].out0 : nullptr; ga.out1[i] = on ? gs[i].out1 : nullptr;
    ga.zero_m0_im[i] = on ? gs[i].zero_m0_im : 0;
  }
  const dim3 pg(ctx->NM, nzb);
  const int srow = o->srow[OzT<TYPE>::anal ? 1 : 0];
  const size_t psm = oz_prep_smem<TYPE>(srow);
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm);
    kern<<<pg, 256, psm, stream>>>(pa, srow);
  };
  switch (o->S) {
    case 2: go(k_oz_prep<TYPE, 2>); break;
    case 3: go(k_oz_prep<TYPE, 3>); break;
    case 4: go(k_oz_prep<TYPE, 4>); break;
    case 5: go(k_oz_prep<TYPE, 5>); break;
    case 6: go(k_oz_prep<TYPE, 6>); break;
    case 7: go(k_oz_prep<TYPE, 7>); break;
    default: go(k_oz_prep<TYPE, 8>); break;
  }
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->dev);
  const int ntile = ctx->NM * 2 * nzb;
  oz_gemm_dispatch<TYPE>(o->S, [&](auto kern) {
    kern<<<std::min(ntile, o->ctas * nsm), OZ_THREADS, o->smem, stream>>>(ga, nzb);
  });
  ctx->launches += 2;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("tensor-core contraction: ") + cudaGetErrorString(e));
  return LSD_OK;
}

template <int TYPE>
int oz_run_all(lsd_ctx* ctx, const std::vector<OzLaunchGroup>& gs, int maxg, cudaStream_t stream) {
  for (size_t i = 0; i < gs.size(); i += maxg) {
    int rc = oz_run<TYPE>(ctx, gs.data() + i, (int)std::min<size_t>(maxg, gs.size() - i), stream);
    if (rc) return rc;
  }
  return LSD_OK;
}

// the branch streams of ctx->stream (created on first use)
OzState::Aux* oz_aux(lsd_ctx* ctx) {
  OzState* o = (OzState*)ctx->oz;
  for (OzState::Aux& x : o->aux)
    if (x.origin == ctx->stream) return &x;
  OzState::Aux x{};
  x.origin = ctx->stream;
  bool ok = cudaEventCreateWithFlags(&x.fork, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < 2 && ok; ++i)
    ok = cudaStreamCreateWithFlags(&x.s[i], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&x.join[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {  // release what was made; the caller reports the failure
    for (int i = 0; i < 2; ++i) {
      if (x.s[i]) cudaStreamDestroy(x.s[i]);
      if (x.join[i]) cudaEventDestroy(x.join[i]);
    }
    if (x.fork) cudaEventDestroy(x.fork);
    return nullptr;
  }
  o->aux.push_back(x);  // the pointer below is used before the next push
  return &o->aux.back();
}

// fn(main, branch 0, branch 1) launches the chains; the branches start after everything
// queued on ctx->stream so far, and ctx->stream waits for both at the end
template <class F>
int oz_forked(lsd_ctx* ctx, F&& fn) {
  OzState::Aux* x = oz_aux(ctx);
  if (!x) return lsd_fail(ctx, LSD_ECUDA, "tensor-core contraction: branch streams");
  cudaStream_t s0 = ctx->stream;
  CUDA_TRY(cudaEventRecord(x->fork, s0));
  for (int i = 0; i < 2; ++i) CUDA_TRY(cudaStreamWaitEvent(x->s[i], x->fork, 0));
  int rc = fn(s0, x->s[0], x->s[1]);
  for (int i = 0; i < 2; ++i) {  // join also after an error, so that no branch is left open
    cudaEventRecord(x->join[i], x->s[i]);
    cudaStreamWaitEvent(s0, x->join[i], 0);
  }
  if (rc) return rc;
  CUDA_TRY(cudaGetLastError());
  return LSD_OK;
}

}  // namespace

// The FP64 group descriptions of the synthesis / analysis launchers, mapped onto the
// tensor-core GEMM types: vector (q,s,t) = P(q) + VEC(s,t); scalar = P; grad3 (dC, C) =
// P(dC) + GRAD(C); grad2 = GRAD; analysis vector (r,th,ph) = Q(r) + ST(th,ph); scalar = Q.
int lsd_ozaki_launch_synth(lsd_ctx* ctx, const SynthGroup* groups, int ngroups) {
  std::vector<OzLaunchGroup> gv, gp, gg;
  for (int i = 0; i < ngroups; ++i) {
    const SynthGroup& G = groups[i];
    switch (G.kind) {
      case SK_VECTOR:
        gp.push_back({G.in[0], nullptr, G.out[0], nullptr, 0});
        gv.push_back({G.in[1], G.in[2], G.out[1], G.out[2], 0});
        break;
      case SK_SCALAR:
        gp.push_back({G.in[0], nullptr, G.out[0], nullptr, 0});
        break;
      case SK_GRAD3:
        gp.push_back({G.in[0], nullptr, G.out[0], nullptr, 0});
        gg.push_back({G.in[1], nullptr, G.out[1], G.out[2], 0});
        break;
      default:  // SK_GRAD2
        gg.push_back({G.in[0], nullptr, G.out[0], G.out[1], 0});
        break;
    }
  }
  // three independent chains (slicing pass -> GEMM each) on forked branches
  return oz_forked(ctx, [&](cudaStream_t s0, cudaStream_t s1, cudaStream_t s2) {
    int rc = oz_run_all<OZ_VEC>(ctx, gv, OZ_MAXG_SYNTH, s0);
    if (!rc) rc = oz_run_all<OZ_P>(ctx, gp, OZ_MAXG_SYNTH, s1);
    if (!rc) rc = oz_run_all<OZ_GRAD>(ctx, gg, OZ_MAXG_SYNTH, s2);
    return rc;
  });
}

int lsd_ozaki_launch_anal(lsd_ctx* ctx, const AnalGroup* groups, int ngroups) {
  std::vector<OzLaunchGroup> gs, gq;
  for (int i = 0; i < ngroups; ++i) {
    const AnalGroup& G = groups[i];
    if (G.kind == AK_VECTOR) {
      gq.push_back({G.in[0], nullptr, G.out[0], nullptr, 0});  // q keeps Im of m = 0
      gs.push_back({G.in[1], G.in[2], G.out[1], G.out[2], 1});
    } else {
      gq.push_back({G.in[0], nullptr, G.out[0], nullptr, 1});
    }
  }
  return oz_forked(ctx, [&](cudaStream_t s0, cudaStream_t s1, cudaStream_t) {
    int rc = oz_run_all<OZ_ST>(ctx, gs, OZ_MAXG_ANAL, s0);
    if (!rc) rc = oz_run_all<OZ_Q>(ctx, gq, OZ_MAXG_ANAL, s1);
    return rc;
  });
}

int* lsd_ozaki_err_flag(lsd_ctx* ctx) { return ((OzState*)ctx->oz)->d_err; }

// The GEMM's tunable tiles: ring stages and CTAs per SM.  A pair is valid when the
// stages (+ 4 KB of static shared memory) fit the shared memory of that many CTAs per SM
// (228 KB per SM, 1 KB reserved per CTA); 256 (ctas = 2) or 512 tensor-memory columns
// each.
bool lsd_ozaki_tiles_ok(int S, int nst, int ctas) {
  if (nst < 2 || nst > OZ_MAXSTAGES || (ctas != 1 && ctas != 2) || S < 2 || S > OZ_MAXS) return false;
  const size_t smem = (size_t)nst * oz_stage_bytes(S) + 4096;  // + static
  return smem * ctas <= (size_t)228 * 1024 - 1024 * ctas;
}
// three stages where two CTAs per SM still fit, else two (at lmax 127, five slices: 2 and
// 3 stages time alike, 4 two per cent slower)
int lsd_ozaki_default_stages(int S) { return lsd_ozaki_tiles_ok(S, 3, 2) ? 3 : 2; }
// the default tiles: the default stages, two CTAs per SM where they fit, else one, so that
// the persistent grid is all resident
void lsd_ozaki_default_tiles(int S, int* nst, int* ctas) {
  *nst = lsd_ozaki_default_stages(S);
  *ctas = lsd_ozaki_tiles_ok(S, *nst, 2) ? 2 : 1;
}
void lsd_ozaki_get_tiles(const lsd_ctx* ctx, int* nst, int* ctas) {
  const OzState* o = (const OzState*)ctx->oz;
  *nst = o ? o->nst : 0;
  *ctas = o ? o->ctas : 0;
}
int lsd_ozaki_set_tiles(lsd_ctx* ctx, int nst, int ctas) {
  OzState* o = (OzState*)ctx->oz;
  if (!o) return LSD_OK;
  if (!lsd_ozaki_tiles_ok(o->S, nst, ctas)) return lsd_fail(ctx, LSD_EARG, "tensor-core GEMM tiles: invalid stages / CTAs");
  o->nst = nst;
  o->ctas = ctas;
  o->smem = (size_t)o->nst * oz_stage_bytes(o->S);
  oz_set_smem<OZ_VEC>(o->S, o->smem); oz_set_smem<OZ_P>(o->S, o->smem); oz_set_smem<OZ_GRAD>(o->S, o->smem);
  oz_set_smem<OZ_ST>(o->S, o->smem); oz_set_smem<OZ_Q>(o->S, o->smem);
  CUDA_TRY(cudaGetLastError());
  return LSD_OK;
}

int lsd_ozaki_check(lsd_ctx* ctx) {
  OzState* o = (OzState*)ctx->oz;
  int err = 0;
  CUDA_TRY(cudaMemcpyAsync(&err, o->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (err) return lsd_fail(ctx, LSD_ECUDA, "tensor-core Legendre contraction: an mbarrier wait timed out");
  return LSD_OK;
}
