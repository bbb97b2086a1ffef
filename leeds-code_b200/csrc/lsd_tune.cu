// lsd_tune.cu -- the autotuner: the phi-FFT radices of the products / c2r / r2c kernels,
// the tensor-core GEMM's ring depth and CTAs per SM, and the banded solves' threads per
// CTA, each chosen by timing its candidates on the context's own configuration.  No
// counterpart in the reference, whose analogue is FFTW's plan search (FFTW_PATIENT in
// tra_precompute, transform.fftw3.F90:76-93).
//
// Timings run on a deterministic pattern written into the state (the kernels' work does
// not depend on the values); the state, the nonlinear terms and the rotation slots are
// restored afterwards, so a tuned context starts like an untuned one.  Choices are kept per
// process and configuration shape, so ensemble members of one shape are timed once.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "lsd_common.cuh"

namespace {

int products_fields(const lsd_config& c) {
  const int nf = c.comp_tstep ? 18 : 15;
  return c.boussinesq ? nf : nf + 2;
}

// the candidates of a configuration, the default of each list first
void tune_space(const lsd_config& c, lsd_tune_space& sp) {
  std::memset(&sp, 0, sizeof(sp));
  const int P2 = c.M * 3 / 2, NM = 2 * ((c.M + 1) / 2);
  int G = 1;
  while (G < 16 && P2 % (2 * G) == 0) G *= 2;
  const int nf = products_fields(c);
  for (int g = G; g >= 4 && sp.nfft < LSD_TUNE_MAX; g /= 2) {
    if (P2 % g) continue;
    const int E = P2 / g;
    if (!lsd_fft_compiled(E, g)) continue;
    if (lsd_products_smem_for(nf, P2, E, g, NM) > 224 * 1024) continue;
    sp.fft_E[sp.nfft] = E;
    sp.fft_G[sp.nfft] = g;
    sp.nfft++;
  }
  if (c.precision == LSD_PREC_OZAKI) {
    const int S = c.ozaki_slices > 0 ? c.ozaki_slices : 7;
    int d = 0, dc = 0;
    lsd_ozaki_default_tiles(S, &d, &dc);
    sp.gemm_stages[0] = d;
    sp.gemm_ctas[0] = dc;
    sp.ngemm = 1;
    for (int ctas = 2; ctas >= 1; --ctas)
      for (int nst = 2; nst <= 4; ++nst) {
        if ((nst == d && ctas == dc) || !lsd_ozaki_tiles_ok(S, nst, ctas) || sp.ngemm >= LSD_TUNE_MAX) continue;
        sp.gemm_stages[sp.ngemm] = nst;
        sp.gemm_ctas[sp.ngemm] = ctas;
        sp.ngemm++;
      }
  }
  const int th[3] = {128, 64, 32};
  for (int t : th) sp.solve_threads[sp.nsolve++] = t;
}

// the selection rule: the fastest, unless it beats the default by less than 2 %
int choose(int n, const double* ms, int dflt) {
  if (n <= 0) return -1;
  if (dflt < 0 || dflt >= n) dflt = 0;
  int best = 0;
  for (int i = 1; i < n; ++i)
    if (ms[i] < ms[best]) best = i;
  return ms[best] < 0.98 * ms[dflt] ? best : dflt;
}

// a deterministic pattern of the magnitude of a state (the timings do not depend on it)
__global__ void k_tune_fill(double* a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long h = (i + 1) * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 32;
    a[i] = 1e-3 * ((double)(h & 0xFFFFF) / (double)0x80000 - 1.0);
  }
}

// the average device time of fn over reps runs (one untimed run first)
template <class F>
int time_ms(lsd_ctx* ctx, F fn, int reps, double* ms) {
  int rc = fn();
  if (rc) return rc;
  CUDA_TRY(cudaEventRecord(ctx->ev0, ctx->stream));
  for (int i = 0; i < reps; ++i)
    if ((rc = fn())) return rc;
  CUDA_TRY(cudaEventRecord(ctx->ev1, ctx->stream));
  CUDA_TRY(cudaEventSynchronize(ctx->ev1));
  float t = 0.f;
  CUDA_TRY(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
  *ms = t / reps;
  return LSD_OK;
}

struct TuneChoice {
  int E, G, nst, ctas, threads;
  double ms_fft, ms_gemm, ms_solve;
};
std::mutex g_tune_mu;
std::map<std::vector<int>, TuneChoice> g_tune_cache;

std::vector<int> shape_key(const lsd_config& c) {
  return {c.L, c.M, c.Mp, c.N, c.Nic, c.KL, c.precision, c.ozaki_slices, c.boussinesq, c.comp_tstep,
          c.device, c.timestep < 0 ? 1 : 0, c.rot_tstep, c.vel_bc};
}

int apply(lsd_ctx* ctx, const TuneChoice& t) {
  ctx->fftE = t.E;
  ctx->fftG = t.G;
  ctx->solve_threads = t.threads;
  if (ctx->oz && t.nst > 0) {
    int rc = lsd_ozaki_set_tiles(ctx, t.nst, t.ctas);
    if (rc) return rc;
  }
  return LSD_OK;
}

}  // namespace

int lsd_autotune(lsd_ctx* ctx) {
  const lsd_config& c = ctx->cfg;
  const std::vector<int> key = shape_key(c);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      int rc = apply(ctx, it->second);
      if (rc) return rc;
      ctx->tuning.tuned = 1;
      ctx->tuning.ms_fft = it->second.ms_fft;
      ctx->tuning.ms_gemm = it->second.ms_gemm;
      ctx->tuning.ms_solve = it->second.ms_solve;
      return LSD_OK;
    }
  }
  lsd_tune_space sp;
  tune_space(c, sp);
  const size_t F = (size_t)ctx->N * ctx->H;
  const int nstate = LSD_NFIELD;
  const size_t Fi = (size_t)ctx->Nic * ctx->H;
  // keep the rotation slots; fill the state with the pattern
  std::vector<double> rot(ROT_NSLOT, 0.0);
  CUDA_TRY(cudaMemcpyAsync(rot.data(), ctx->d_rot, sizeof(double) * ROT_NSLOT, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  k_tune_fill<<<592, 256, 0, ctx->stream>>>((double*)ctx->d_state, 2 * nstate * F);
  CUDA_TRY(cudaGetLastError());
  const int reps = 3;
  TuneChoice ch{ctx->fftE, ctx->fftG, 0, 0, ctx->solve_threads, 0.0, 0.0, 0.0};
  // phi-FFT radices: one evaluation each
  {
    std::vector<double> ms(sp.nfft, 0.0);
    for (int i = 0; i < sp.nfft; ++i) {
      ctx->fftE = sp.fft_E[i];
      ctx->fftG = sp.fft_G[i];
      int rc = time_ms(ctx, [&]() { return lsd_eval(ctx); }, reps, &ms[i]);
      if (rc) return rc;
    }
    const int k = choose(sp.nfft, ms.data(), 0);
    ch.E = sp.fft_E[k];
    ch.G = sp.fft_G[k];
    ch.ms_fft = ms[k];
    ctx->fftE = ch.E;
    ctx->fftG = ch.G;
  }
  // tensor-core GEMM tiles: one evaluation each
  if (ctx->oz && sp.ngemm > 0) {
    std::vector<double> ms(sp.ngemm, 0.0);
    for (int i = 0; i < sp.ngemm; ++i) {
      int rc = lsd_ozaki_set_tiles(ctx, sp.gemm_stages[i], sp.gemm_ctas[i]);
      if (!rc) rc = time_ms(ctx, [&]() { return lsd_eval(ctx); }, reps, &ms[i]);
      if (rc) return rc;
    }
    const int k = choose(sp.ngemm, ms.data(), 0);
    ch.nst = sp.gemm_stages[k];
    ch.ctas = sp.gemm_ctas[k];
    ch.ms_gemm = ms[k];
    int rc = lsd_ozaki_set_tiles(ctx, ch.nst, ch.ctas);
    if (rc) return rc;
  }
  // banded solves: one predictor solve each (the state it leaves is discarded below)
  {
    std::vector<double> ms(sp.nsolve, 0.0);
    for (int i = 0; i < sp.nsolve; ++i) {
      ctx->solve_threads = sp.solve_threads[i];
      int rc = time_ms(ctx, [&]() { return lsd_pred(ctx); }, reps, &ms[i]);
      if (rc) return rc;
    }
    const int k = choose(sp.nsolve, ms.data(), 0);
    ch.threads = sp.solve_threads[k];
    ch.ms_solve = ms[k];
    ctx->solve_threads = ch.threads;
  }
  // back to the state of a new context
  CUDA_TRY(cudaMemsetAsync(ctx->d_state, 0, sizeof(cplx) * nstate * F, ctx->stream));
  CUDA_TRY(cudaMemsetAsync(ctx->d_nl, 0, sizeof(cplx) * nstate * F, ctx->stream));
  CUDA_TRY(cudaMemsetAsync(ctx->d_sv, 0, sizeof(cplx) * nstate * F, ctx->stream));
  if (ctx->Nic > 1) {
    CUDA_TRY(cudaMemsetAsync(ctx->d_icstate, 0, sizeof(cplx) * 2 * Fi, ctx->stream));
    CUDA_TRY(cudaMemsetAsync(ctx->d_icsv, 0, sizeof(cplx) * 2 * Fi, ctx->stream));
  }
  CUDA_TRY(cudaMemcpyAsync(ctx->d_rot, rot.data(), sizeof(double) * ROT_NSLOT, cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (ctx->oz) {
    int rc = lsd_ozaki_check(ctx);
    if (rc) return rc;
  }
  ctx->tuning.tuned = 1;
  ctx->tuning.ms_fft = ch.ms_fft;
  ctx->tuning.ms_gemm = ch.ms_gemm;
  ctx->tuning.ms_solve = ch.ms_solve;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = ch;
  return LSD_OK;
}

extern "C" {

int lsd_tune_candidates(const lsd_config* cfg, lsd_tune_space* out) {
  if (!cfg || !out) return LSD_EARG;
  tune_space(*cfg, *out);
  return out->nfft > 0 ? LSD_OK : LSD_EARG;
}

int lsd_tune_choose(int n, const double* ms, int dflt) { return (!ms || n <= 0) ? -1 : choose(n, ms, dflt); }

int lsd_get_tuning(const lsd_ctx* ctx, lsd_tuning* out) {
  if (!ctx || !out) return LSD_EARG;
  *out = ctx->tuning;
  out->fft_E = ctx->fftE;
  out->fft_G = ctx->fftG;
  int nst = 0, ctas = 0;
  if (ctx->oz) lsd_ozaki_get_tiles(ctx, &nst, &ctas);
  out->gemm_stages = nst;
  out->gemm_ctas_per_sm = ctas;
  out->solve_threads = ctx->solve_threads;
  return LSD_OK;
}

int lsd_set_tuning(lsd_ctx* ctx, const lsd_tuning* in) {
  if (!ctx || !in) return LSD_EARG;
  lsd_tune_space sp;
  tune_space(ctx->cfg, sp);
  bool fft_ok = false, th_ok = false;
  for (int i = 0; i < sp.nfft; ++i) fft_ok |= sp.fft_E[i] == in->fft_E && sp.fft_G[i] == in->fft_G;
  for (int i = 0; i < sp.nsolve; ++i) th_ok |= sp.solve_threads[i] == in->solve_threads;
  if (!fft_ok) return lsd_fail(ctx, LSD_EARG, "lsd_set_tuning: (fft_E, fft_G) is not a candidate of this configuration");
  if (!th_ok) return lsd_fail(ctx, LSD_EARG, "lsd_set_tuning: solve_threads must be 32, 64 or 128");
  CUDA_TRY(cudaSetDevice(ctx->dev));
  if (ctx->oz) {
    int rc = lsd_ozaki_set_tiles(ctx, in->gemm_stages, in->gemm_ctas_per_sm);
    if (rc) return rc;
  }
  ctx->fftE = in->fft_E;
  ctx->fftG = in->fft_G;
  ctx->solve_threads = in->solve_threads;
  if (ctx->g_step) {  // the step graph holds the old launch shapes: captured again at the next step
    cudaGraphExecDestroy(ctx->g_step);
    ctx->g_step = nullptr;
  }
  return LSD_OK;
}

}  // extern "C"
