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
