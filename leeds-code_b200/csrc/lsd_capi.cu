// lsd_capi.cu -- the extern "C" entry points of include/lsd_b200.h.
//
// Host-side control mirrors the reference's driver: initialise (main.F90:220-400),
// the main loop (main.F90:100-164) with tim_check_cgce (timestep.F90:744-830), and the
// state refresh for output.  Every entry point returns a status; nothing aborts.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "lsd_common.cuh"

static_assert(sizeof(PcState) == sizeof(lsd_pc_state), "lsd_pc_state mirrors PcState");

int lsd_fail(lsd_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

namespace {


void free_ctx(lsd_ctx* ctx) {
  if (!ctx) return;
  if (ctx->dev >= 0) cudaSetDevice(ctx->dev);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->g_step) cudaGraphExecDestroy(ctx->g_step);
  for (cudaStream_t cs : ctx->cap_stream)
    if (cs) cudaStreamDestroy(cs);
  for (lsd_ctx::Aux& x : ctx->eval_aux) {
    for (int i = 0; i < 2; ++i) {
      cudaStreamDestroy(x.s[i]);
      cudaEventDestroy(x.join[i]);
    }
    cudaEventDestroy(x.fork);
  }
  lsd_ozaki_free(ctx);
  void* ptrs[] = {ctx->d_sblk_l, ctx->d_sblk_nh, ctx->d_aperm, ctx->d_l, ctx->d_m, ctx->d_s, ctx->d_mc, ctx->d_mstart, ctx->d_mlen, ctx->d_thm, ctx->d_bin2c, ctx->d_lm2nh,
                  ctx->d_leg, ctx->d_gp, ctx->d_gw, ctx->d_sn, ctx->d_sn1, ctx->d_tw2, ctx->d_twh, ctx->d_r,
                  ctx->d_dr, ctx->d_r1dr, ctx->d_radlap, ctx->d_intr2dr, ctx->d_lu, ctx->d_lus, ctx->d_y, ctx->d_yt,
                  ctx->d_ipiv, ctx->d_ipivs, ctx->d_info, ctx->d_gre, ctx->d_gret, ctx->d_invg, ctx->d_state, ctx->d_nl,
                  ctx->d_sv, ctx->d_spec, ctx->d_four, ctx->d_phys, ctx->d_red, ctx->d_cpart, ctx->d_ref, ctx->d_laps,
                  ctx->d_compr1dr, ctx->d_wts, ctx->d_ones, ctx->d_cfl, ctx->d_icr, ctx->d_icdr, ctx->d_icradlap,
                  ctx->d_icr1dr, ctx->d_icintr2dr, ctx->d_icwts, ctx->d_icref, ctx->d_iclaps, ctx->d_iccompr1dr,
                  ctx->d_icyt, ctx->d_icstate, ctx->d_icsv, ctx->d_rot, ctx->d_gwP0, ctx->d_grescr,
                  ctx->d_pc, ctx->d_opfail};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (ctx->h_pin) cudaFreeHost(ctx->h_pin);
  if (ctx->h_red) cudaFreeHost(ctx->h_red);
  if (ctx->h_pc) cudaFreeHost(ctx->h_pc);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  if (ctx->d_stage) cudaFree(ctx->d_stage);
  for (int k = 0; k < 2; ++k) {
    if (ctx->ev_staged[k]) cudaEventDestroy(ctx->ev_staged[k]);
    if (ctx->ev_committed[k]) cudaEventDestroy(ctx->ev_committed[k]);
  }
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->stream && ctx->owns_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

template <class T>
int dalloc(lsd_ctx* ctx, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return LSD_OK;
}

// Host-to-device copies that kernels on the context's stream read go on that stream: a
// plain cudaMemcpy runs on the legacy default stream, which a non-blocking stream does not
// wait for, and from pageable memory it returns once the data is staged, before its DMA
// has landed.  cudaMemcpyAsync from pageable memory also stages before returning, so the
// host buffer may be reused at once.
template <class T>
int upload(lsd_ctx* ctx, T* d, const std::vector<T>& h) {
  CUDA_TRY(cudaMemcpyAsync(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, ctx->stream));
  return LSD_OK;
}
int h2d(lsd_ctx* ctx, void* d, const void* h, size_t bytes) {
  CUDA_TRY(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return LSD_OK;
}


// harmonic layout: _loop_setlm (parallel.h_template:54-80), _loop_sumth (:85-100)
void build_layout(lsd_ctx* c) {
  c->hl.assign(c->H, 0); c->hm.assign(c->H, 0); c->hs.assign(c->H, 0); c->mcount.assign(c->H, 0);
  int nh = -1;
  for (int j = 1; j <= c->Hc; ++j)
    for (int i = 1; i <= c->Hr; ++i) {
      int m = j - 1, l = m * c->Mp + i - 1;
      if (l >= c->L) { m = 2 * c->Hc - j; l = c->L - c->Hr + i - 1; }
      ++nh;
      c->hl[nh] = l; c->hm[nh] = m * c->Mp; c->hs[nh] = (l + m * c->Mp) % 2;
    }
  c->thm.assign(c->NM, 0);
  c->mstart.assign(c->NM, 0);
  c->mlen.assign(c->NM, 0);
  int m = -1, m_ = -1;
  for (nh = 0; nh < c->H; ++nh) {
    int m__ = m_;
    m_ = c->hm[nh];
    if (m_ != m__) { ++m; c->thm[m] = m_ / c->Mp; c->mstart[m] = nh; }
    c->mcount[nh] = m;
    c->mlen[m]++;
  }
}

// radix plan for the complex FFT of length P2 = 3^a 2^b

void pack_spec(const lsd_ctx* c, const double* re, const double* im, double* out) {  // spec (H,N)
  size_t T = (size_t)c->N * c->H;
  for (size_t i = 0; i < T; ++i) { out[2 * i] = re[i]; out[2 * i + 1] = im[i]; }
}
void unpack_spec(const lsd_ctx* c, const double* in, double* re, double* im) {
  size_t T = (size_t)c->N * c->H;
  for (size_t i = 0; i < T; ++i) { re[i] = in[2 * i]; im[i] = in[2 * i + 1]; }
}

int ensure_phys(lsd_ctx* ctx, int nslots) {
  if (ctx->nphys >= nslots) return LSD_OK;
  if (ctx->d_phys) { cudaFree(ctx->d_phys); ctx->d_phys = nullptr; }
  int rc = dalloc(ctx, &ctx->d_phys, (size_t)nslots * ctx->N * ctx->Ph * ctx->Th);
  if (rc) return rc;
  ctx->nphys = nslots;
  return LSD_OK;
}

int time_begin(lsd_ctx* ctx) {
  CUDA_TRY(cudaEventRecord(ctx->ev0, ctx->stream));
  return LSD_OK;
}
int time_end(lsd_ctx* ctx) {
  CUDA_TRY(cudaEventRecord(ctx->ev1, ctx->stream));
  CUDA_TRY(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->last_ms = ms;
  if (ctx->oz) return lsd_ozaki_check(ctx);
  return LSD_OK;
}

// the host copy of the loop control (lsd_ctx fields) as the shared PcState and back
PcState pc_get(const lsd_ctx* c) {
  PcState s;
  s.t = c->t; s.dt = c->dt; s.dterr = c->dterr; s.corr_dt = c->corr_dt; s.lasterr = c->lasterr;
  s.cfl_dt = c->cfl_dt; s.it = c->it; s.step = c->step; s.pcn = c->tim_pcn; s.pad_ = 0;
  return s;
}
void pc_put(lsd_ctx* c, const PcState& s) {
  c->t = s.t; c->dt = s.dt; c->dterr = s.dterr; c->corr_dt = s.corr_dt; c->lasterr = s.lasterr;
  c->cfl_dt = s.cfl_dt; c->it = s.it; c->step = s.step; c->tim_pcn = s.pcn;
}
PcParams pc_params(const lsd_config& g) {
  PcParams p;
  p.timestep = g.timestep; p.dterr = g.dterr; p.courant = g.courant; p.corr_upper = g.corr_upper;
  p.corr_lower = g.corr_lower; p.control = g.time_step_control; p.pad_ = 0;
  return p;
}

// tim_check_cgce (timestep.F90:744-830) on the host copy; LSD_ENOTCONVERGED when it gives up
int check_cgce(lsd_ctx* c) {
  PcState s = pc_get(c);
  const bool ok = pc_check_cgce(s, pc_params(c->cfg));
  pc_put(c, s);
  return ok ? LSD_OK : LSD_ENOTCONVERGED;
}

// queue the copy of the corrector's sums of squares (and the tensor-core error flag) to
// the pinned mirror; finish_corrector_host reads them once the stream got there
int enqueue_corrector_readback(lsd_ctx* ctx) {
  CUDA_TRY(cudaMemcpyAsync(ctx->h_red, ctx->d_red, sizeof(double) * 8, cudaMemcpyDeviceToHost, ctx->stream));
  int* oz_err = (int*)(ctx->h_red + LSD_HRED_OZERR);
  *oz_err = 0;
  if (ctx->oz) CUDA_TRY(cudaMemcpyAsync(oz_err, lsd_ozaki_err_flag(ctx), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  return LSD_OK;
}

// tim_dterr (timestep.F90:715-737) from the corrector's sums of squares r[0..7], added to
// d in the reference's field order
__host__ __device__ inline double dterr_sum(double d, const double* r, bool comp) {
  d = d + sqrt(r[0]);  // vel Tor
  d = d + sqrt(r[1]);  // vel Pol
  d = d + sqrt(r[2]);  // codensity
  if (comp) d = d + sqrt(r[3]);
  d = d + sqrt(r[4]);  // mag Tor
  d = d + sqrt(r[5]);  // inner-core Tor
  d = d + sqrt(r[6]);  // mag Pol
  d = d + sqrt(r[7]);  // inner-core Pol
  return d;
}

// form tim_dterr from the mirrored sums of squares
int finish_corrector_host(lsd_ctx* ctx) {
  const int* oz_err = (const int*)(ctx->h_red + LSD_HRED_OZERR);
  if (*oz_err) return lsd_fail(ctx, LSD_ECUDA, "tensor-core Legendre contraction: an mbarrier wait timed out");
  const double d = dterr_sum(ctx->dterr, ctx->h_red, ctx->cfg.comp_tstep != 0);
  ctx->dterr = d;
  if (!std::isfinite(d)) return lsd_fail(ctx, LSD_ENONFINITE, "non-finite corrector norm (state diverged)");
  return LSD_OK;
}

int finish_corrector(lsd_ctx* ctx) {
  int rc = enqueue_corrector_readback(ctx);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return finish_corrector_host(ctx);
}

// ---- the one-graph step -------------------------------------------------------------
// Control kernels (one thread each) of the graph lsd_step launches.  The loop state lives
// in the context's PcDev; the WHILE / IF conditions are set with cudaGraphSetConditional.
// Every loop has a hard iteration cap besides the reference's own limits, so the graph
// always ends: the step loop stops after the call's nsteps iterations, the corrector loop
// after 64 correctors of one step (tim_check_cgce gives up after 11).
constexpr int PC_MAX_CORR = 64;

// start of the call: the host has uploaded the state, steps_left = nsteps, counters zero
__global__ void k_pc_begin(PcDev* pc, cudaGraphConditionalHandle h_steps) {
  cudaGraphSetConditional(h_steps, pc->steps_left > 0 && pc->status == LSD_OK ? 1u : 0u);
}

// d_timestep < 0, after the step's first evaluation: non_maxtstep's tim_cfl_dt and
// tim_new_tstep (main.F90:126-134); the IF node that follows rebuilds the operators when
// dt changed
__global__ void k_pc_newdt(PcDev* pc, const double* cfl, PcParams p, cudaGraphConditionalHandle h_rebuild) {
  pc->s.cfl_dt = *cfl;
  const bool nd = pc_new_tstep(pc->s, p);
  if (nd) pc->rebuilds++;
  cudaGraphSetConditional(h_rebuild, nd ? 1u : 0u);
}

// after the predictor (main.F90:136-147): tim_it = 1, and the corrector loop starts
__global__ void k_pc_pred(PcDev* pc, cudaGraphConditionalHandle h_corr) {
  pc->s.it = 1;
  pc->evaluations++;
  pc->iters = 0;
  cudaGraphSetConditional(h_corr, pc->status == LSD_OK ? 1u : 0u);
}

// after a corrector (main.F90:148-155): tim_dterr, tim_check_cgce, and at the end of the
// step tim_t += tim_dt, tim_step += 1 (main.F90:158-161)
__global__ void k_pc_corr(PcDev* pc, const double* red, int comp, const int* oz_err, PcParams p,
                          cudaGraphConditionalHandle h_corr) {
  pc->evaluations++;
  pc->correctors++;
  pc->iters++;
  const double d = dterr_sum(0.0, red, comp != 0);
  pc->s.dterr = d;
  pc->last_dterr = d;
  int st = pc->status;
  if (st == LSD_OK) {
    if (oz_err && *oz_err) st = LSD_ECUDA;
    else if (!isfinite(d)) st = LSD_ENONFINITE;
    else if (!pc_check_cgce(pc->s, p)) st = LSD_ENOTCONVERGED;
    else if (pc->s.it == 0) {
      pc->s.t = pc->s.t + pc->s.dt;
      pc->s.step = pc->s.step + 1;
      pc->steps_done++;
      pc->steps_left--;
    } else if (pc->iters >= PC_MAX_CORR) st = LSD_ENOTCONVERGED;
  }
  pc->status = st;
  cudaGraphSetConditional(h_corr, st == LSD_OK && pc->s.it != 0 ? 1u : 0u);
}

// end of a step-loop iteration
__global__ void k_pc_end(PcDev* pc, cudaGraphConditionalHandle h_steps) {
  pc->loops++;
  const bool more = pc->status == LSD_OK && pc->steps_left > 0 && pc->loops < pc->nsteps;
  cudaGraphSetConditional(h_steps, more ? 1u : 0u);
}

// Adds a conditional node of `type` on handle h at the current point of the capture on
// `s` and returns its body graph; the capture on s continues after the node.
int cap_conditional(lsd_ctx* ctx, cudaStream_t s, cudaGraphConditionalNodeType type,
                    cudaGraphConditionalHandle h, cudaGraph_t* body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  CUDA_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive) return lsd_fail(ctx, LSD_ECUDA, "graph capture: stream not capturing");
  cudaGraphNodeParams prm = {};
  prm.type = cudaGraphNodeTypeConditional;
  prm.conditional.handle = h;
  prm.conditional.type = type;
  prm.conditional.size = 1;
  cudaGraphNode_t node;
  CUDA_TRY(cudaGraphAddNode(&node, g, deps, nd, &prm));
  *body = prm.conditional.phGraph_out[0];
  CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  return LSD_OK;
}

// a conditional handle of the graph being captured on s (reset to 0 at every launch)
int cap_handle(lsd_ctx* ctx, cudaStream_t s, cudaGraphConditionalHandle* h) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  CUDA_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, nullptr, nullptr));
  CUDA_TRY(cudaGraphConditionalHandleCreate(h, g, 0, cudaGraphCondAssignDefault));
  return LSD_OK;
}

// Captures into `body` on capture stream k whatever fn launches on ctx->stream.
template <class F>
int cap_body(lsd_ctx* ctx, int k, cudaGraph_t body, F fn) {
  cudaStream_t cs = ctx->cap_stream[k], saved = ctx->stream;
  CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  ctx->stream = cs;
  int rc = fn();
  ctx->stream = saved;
  cudaGraph_t out = nullptr;
  cudaError_t e = cudaStreamEndCapture(cs, &out);
  if (rc) return rc;
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("graph body capture: ") + cudaGetErrorString(e));
  return LSD_OK;
}

// The whole of lsd_step (structure in include/lsd_b200.h at lsd_step), captured on
// ctx->stream, which must be capturing already (into this context's graph, or into the
// graph of an ensemble); sets the kernel counts of the sections.
int capture_step_into(lsd_ctx* ctx) {
  for (cudaStream_t& cs : ctx->cap_stream)
    if (!cs) CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  const PcParams prm = pc_params(ctx->cfg);
  const bool vardt = ctx->cfg.timestep < 0;
  PcDev* pc = ctx->d_pc;
  const int* ozerr = ctx->oz ? lsd_ozaki_err_flag(ctx) : nullptr;
  cudaStream_t s0 = ctx->stream;
  const long long l0 = ctx->launches;
  long long loop = 0, rebuild = 0, corr = 0;
  int rc = LSD_OK;
  cudaGraphConditionalHandle h_steps = 0;
  cudaGraph_t b_steps = nullptr;
  if (!rc) rc = cap_handle(ctx, s0, &h_steps);
  if (!rc) {
    k_pc_begin<<<1, 1, 0, s0>>>(pc, h_steps);
    rc = cap_conditional(ctx, s0, cudaGraphCondTypeWhile, h_steps, &b_steps);
  }
  if (!rc) rc = cap_body(ctx, 0, b_steps, [&]() {
    cudaStream_t s1 = ctx->stream;
    const long long a = ctx->launches;
    int r = lsd_eval(ctx);
    if (!r && vardt) {
      cudaGraphConditionalHandle h_rb = 0;
      cudaGraph_t b_rb = nullptr;
      if (!r) r = cap_handle(ctx, s1, &h_rb);
      if (!r) {
        k_pc_newdt<<<1, 1, 0, s1>>>(pc, ctx->d_cfl + 2 * ctx->N, prm, h_rb);
        ++ctx->launches;
        r = cap_conditional(ctx, s1, cudaGraphCondTypeIf, h_rb, &b_rb);
      }
      if (!r) r = cap_body(ctx, 1, b_rb, [&]() {
        const long long b = ctx->launches;
        int q = lsd_launch_operator_build(ctx, &pc->s.dt, &pc->status);
        rebuild = ctx->launches - b;
        return q;
      });
    }
    if (!r) r = lsd_pred(ctx);
    cudaGraphConditionalHandle h_corr = 0;
    cudaGraph_t b_corr = nullptr;
    if (!r) r = cap_handle(ctx, s1, &h_corr);
    if (!r) {
      k_pc_pred<<<1, 1, 0, s1>>>(pc, h_corr);
      ++ctx->launches;
      r = cap_conditional(ctx, s1, cudaGraphCondTypeWhile, h_corr, &b_corr);
    }
    if (!r) r = cap_body(ctx, 1, b_corr, [&]() {
      const long long b = ctx->launches;
      int q = lsd_eval(ctx);
      if (!q) q = lsd_corr(ctx);
      if (!q) {
        k_pc_corr<<<1, 1, 0, ctx->stream>>>(pc, ctx->d_red, ctx->cfg.comp_tstep, ozerr, prm, h_corr);
        ++ctx->launches;
      }
      corr = ctx->launches - b;
      return q;
    });
    if (!r) {
      k_pc_end<<<1, 1, 0, s1>>>(pc, h_steps);
      ++ctx->launches;
    }
    loop = ctx->launches - a - corr - rebuild;
    return r;
  });
  ctx->launches = l0;
  if (rc) return rc;
  ctx->k_begin = 1;
  ctx->k_loop = loop;
  ctx->k_rebuild = rebuild;
  ctx->k_corr = corr;
  return LSD_OK;
}

int instantiate(lsd_ctx* ctx, cudaGraph_t g, cudaGraphExec_t* out) {
  cudaError_t e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("step graph: ") + cudaGetErrorString(e));
  return LSD_OK;
}

// lsd_step's graph of one context
int capture_step(lsd_ctx* ctx) {
  CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
  int rc = capture_step_into(ctx);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  return instantiate(ctx, g, &ctx->g_step);
}

// A step begun by lsd_predictor / lsd_corrector calls (tim_it != 0): its remaining
// correctors on the host, with tim_check_cgce after each (main.F90:148-161).
int finish_open_step(lsd_ctx* ctx, int* corr, int* evals, double* last) {
  while (ctx->it != 0) {
    ctx->dterr = 0.0;
    int rc = lsd_eval(ctx);
    if (!rc) rc = lsd_corr(ctx);
    if (!rc) rc = finish_corrector(ctx);
    if (rc) return rc;
    ++*corr;
    *evals += 1;
    *last = ctx->dterr;
    if ((rc = check_cgce(ctx))) return lsd_fail(ctx, rc, "tim_check_cgce: corrector iterations did not converge");
  }
  ctx->t = ctx->t + ctx->dt;
  ctx->step = ctx->step + 1;
  return LSD_OK;
}

// The loop state of a call of nsteps steps into the control block (on stream s)
int pc_upload(lsd_ctx* ctx, int nsteps, cudaStream_t s) {
  PcDev* h = ctx->h_pc;
  std::memset(h, 0, sizeof(PcDev));
  h->s = pc_get(ctx);
  h->s.dterr = 0.0;
  h->steps_left = nsteps;
  h->nsteps = nsteps;
  h->status = LSD_OK;
  CUDA_TRY(cudaMemcpyAsync(ctx->d_pc, h, sizeof(PcDev), cudaMemcpyHostToDevice, s));
  return LSD_OK;
}
int pc_download(lsd_ctx* ctx, cudaStream_t s) {
  CUDA_TRY(cudaMemcpyAsync(ctx->h_pc, ctx->d_pc, sizeof(PcDev), cudaMemcpyDeviceToHost, s));
  return LSD_OK;
}

// Queue one launch of the step graph for nsteps steps: the loop state goes up with it and
// comes back into the pinned mirror (read by step_graph_finish after the stream is done).
int step_graph_enqueue(lsd_ctx* ctx, int nsteps) {
  if (!ctx->g_step) {
    int rc = capture_step(ctx);
    if (rc) return rc;
  }
  int rc = pc_upload(ctx, nsteps, ctx->stream);
  if (rc) return rc;
  CUDA_TRY(cudaGraphLaunch(ctx->g_step, ctx->stream));
  return pc_download(ctx, ctx->stream);
}

// after the stream passed the graph: the loop state back into the context, the counts of
// the call, and its outcome
int step_graph_finish(lsd_ctx* ctx, int* done, int* corr, int* evals, double* last, long long* kernels) {
  const PcDev& h = *ctx->h_pc;
  const bool dt_changed = h.rebuilds > 0;
  pc_put(ctx, h.s);
  ctx->dterr = 0.0;
  *done += h.steps_done;
  *corr += h.correctors;
  *evals += h.evaluations;
  if (h.correctors > 0) *last = h.last_dterr;
  *kernels += ctx->k_begin + (long long)h.loops * ctx->k_loop + (long long)h.correctors * ctx->k_corr +
              (long long)h.rebuilds * ctx->k_rebuild;
  if (dt_changed) ctx->op_dt = ctx->dt;
  switch (h.status) {
    case LSD_OK: return LSD_OK;
    case LSD_ENOTCONVERGED: return lsd_fail(ctx, LSD_ENOTCONVERGED, "tim_check_cgce: corrector iterations did not converge");
    case LSD_ENONFINITE: return lsd_fail(ctx, LSD_ENONFINITE, "non-finite corrector norm (state diverged)");
    case LSD_ESINGULAR: return lsd_fail(ctx, LSD_ESINGULAR, "operator rebuild after a dt change: zero pivot or singular influence matrix");
    default: return lsd_fail(ctx, LSD_ECUDA, "tensor-core Legendre contraction: an mbarrier wait timed out");
  }
}

}  // namespace

extern "C" {

int lsd_config_default(lsd_config* c) {
  if (!c) return LSD_EARG;
  std::memset(c, 0, sizeof(*c));
  c->L = 64; c->M = 16; c->Mp = 4; c->N = 64; c->Nic = 1; c->KL = 3;
  c->vel_bc = 1; c->cod_bc = 1; c->comp_bc = 1; c->time_step_control = 2;
  c->boussinesq = 1; c->vel_tstep = 1; c->cod_tstep = 1; c->comp_tstep = 0; c->mag_tstep = 1;
  c->precision = LSD_PREC_FP64; c->device = 0; c->ozaki_slices = 0;
  c->rratio = 0.35; c->alpha = -1.0; c->Ra = 6.5e4; c->Ra_comp = 1.0; c->Pr = 1.0; c->Sc = 1.0;
  c->Pm = 5.0; c->E = 1.0e-3; c->Hyp = 0.0;
  c->implicit = 0.6; c->timestep = -5e-5; c->dterr = 0.025; c->courant = (double)0.8f;
  c->corr_upper = 0.020; c->corr_lower = 0.00200;
  c->source = 0.0; c->source_comp = 0.0; c->qi = 0.0; c->qo = -1.0; c->qi_comp = 0.0; c->qo_comp = -1.0;
  return LSD_OK;
}

// why the last lsd_create of this thread failed (lsd_last_error(NULL) returns it)
static thread_local std::string t_create_err;

int lsd_create(const lsd_config* cfg, lsd_ctx** out) {
  t_create_err.clear();
  if (!cfg || !out) { t_create_err = "lsd_create: null argument"; return LSD_EARG; }
  *out = nullptr;
  lsd_ctx* ctx = new (std::nothrow) lsd_ctx();
  if (!ctx) return LSD_ENOMEM;
  ctx->cfg = *cfg;
  ctx->dev = -1;
  const lsd_config& c = *cfg;
  ctx->L = c.L; ctx->M = c.M; ctx->Mp = c.Mp; ctx->N = c.N; ctx->KL = c.KL;
  ctx->Nic = c.Nic; ctx->NL = c.N + c.Nic - 1;
  // par_precompute (parameters.F90_template:274-288) and this library's scope
  std::string why;
  if (c.L < 2 || c.M < 2 || c.Mp < 1 || c.N < 2 * c.KL + 2 || c.KL < 2 || c.KL > LSD_MAX_KL) why = "bad resolution";
  else if (c.L <= (c.M - 1) * c.Mp) why = "set L > (M-1)*Mp";
  else if (c.M % 2 == 1) why = "if(M>1) set M even";
  else if (c.KL > 6) why = "the timestep kernels are built for stencil half-widths KL = 2..6";
  else if (c.Nic < 1) why = "Nic must be >= 1";
  else if (c.Nic > 1 && (c.Nic < 2 * c.KL + 1 || c.Nic > c.N))
    why = "a conducting inner core needs 2 KL + 1 <= Nic <= N radial points";
  else if (c.Nic > 1 && !c.boussinesq)
    why = "a conducting inner core is supported for the Boussinesq equations";
  else if (c.Nic > 1 && c.vel_bc > 2)
    why = "a conducting inner core needs a no-slip inner wall (i_vel_bc 1 or 2)";
  else if (c.rot_tstep && !c.boussinesq) why = "inner-core rotation is supported for the Boussinesq equations";
  else if (c.timestep == 0.0) why = "d_timestep must be > 0 (fixed) or < 0 (CFL / corrector controlled)";
  else if (!c.vel_tstep || !c.cod_tstep || !c.mag_tstep) why = "velocity, codensity and field must all be stepped";
  else if (c.precision != LSD_PREC_FP64 && c.precision != LSD_PREC_OZAKI) why = "unknown precision";
  else if (c.precision == LSD_PREC_OZAKI && c.ozaki_slices != 0 && (c.ozaki_slices < 2 || c.ozaki_slices > 8))
    why = "ozaki_slices must be 0 (default) or 2..8";
  if (!why.empty()) { t_create_err = why; int rc = lsd_fail(ctx, LSD_EARG, why); free_ctx(ctx); return rc; }
  ctx->Ma = c.M * 3 / 2;
  ctx->H = c.L * c.M - c.Mp * (c.M - 1) * c.M / 2;
  ctx->Th = c.L * 3 / 2;
  ctx->Th2 = (ctx->Th + 1) / 2;
  ctx->Ph = ctx->Ma * 2;
  ctx->Hc = (c.M + 1) / 2;
  ctx->Hr = ctx->H / ctx->Hc;
  ctx->NM = 2 * ctx->Hc;
  ctx->P2 = ctx->Ma;
  ctx->dt = c.timestep < 0 ? -c.timestep : c.timestep;  // d_timestep < 0: |d_timestep| until lsd_set_time
  ctx->HB = (ctx->Th2 + 1) / 2;
  if (!lsd_fft_plan(ctx)) {
    t_create_err = "phi FFT length 3M/2 not supported";
    int rc = lsd_fail(ctx, LSD_EARG, t_create_err);
    free_ctx(ctx);
    return rc;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || c.device < 0 || c.device >= ndev) {
    t_create_err = ndev == 0 ? "no CUDA device" : "device index out of range";
    free_ctx(ctx);
    return LSD_ECUDA;
  }
  ctx->dev = c.device;
  int rc = LSD_OK;
#define TRY(x) do { rc = (x); if (rc) { free_ctx(ctx); return rc; } } while (0)
#define CTRY(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { free_ctx(ctx); return LSD_ECUDA; } } while (0)
  CTRY(cudaSetDevice(ctx->dev));
  CTRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  ctx->owns_stream = true;
  CTRY(cudaEventCreate(&ctx->ev0));
  CTRY(cudaEventCreate(&ctx->ev1));
  build_layout(ctx);
  const int H = ctx->H, N = ctx->N, L = ctx->L, KL = ctx->KL, Th = ctx->Th, Th2 = ctx->Th2, NM = ctx->NM;
  std::vector<int> lm2nh((size_t)ctx->M * L, -1);
  for (int nh = 0; nh < H; ++nh) lm2nh[(size_t)(ctx->hm[nh] / ctx->Mp) * L + ctx->hl[nh]] = nh;
  TRY(dalloc(ctx, &ctx->d_l, H)); TRY(upload(ctx, ctx->d_l, ctx->hl));
  TRY(dalloc(ctx, &ctx->d_m, H)); TRY(upload(ctx, ctx->d_m, ctx->hm));
  TRY(dalloc(ctx, &ctx->d_s, H)); TRY(upload(ctx, ctx->d_s, ctx->hs));
  TRY(dalloc(ctx, &ctx->d_mc, H)); TRY(upload(ctx, ctx->d_mc, ctx->mcount));
  TRY(dalloc(ctx, &ctx->d_mstart, NM)); TRY(upload(ctx, ctx->d_mstart, ctx->mstart));
  TRY(dalloc(ctx, &ctx->d_mlen, NM)); TRY(upload(ctx, ctx->d_mlen, ctx->mlen));
  TRY(dalloc(ctx, &ctx->d_thm, NM)); TRY(upload(ctx, ctx->d_thm, ctx->thm));
  {  // FFT bin -> m-counter (var_Th%m is a permutation of the bins 0..M-1)
    std::vector<int> b2c(ctx->M, 0);
    for (int c = 0; c < NM; ++c)
      if (ctx->thm[c] >= 0 && ctx->thm[c] < ctx->M) b2c[ctx->thm[c]] = c;
    TRY(dalloc(ctx, &ctx->d_bin2c, b2c.size())); TRY(upload(ctx, ctx->d_bin2c, b2c));
  }
  TRY(dalloc(ctx, &ctx->d_lm2nh, lm2nh.size())); TRY(upload(ctx, ctx->d_lm2nh, lm2nh));
  {  // analysis thread order per folded column: (m-counter, parity)-sorted harmonics
    std::vector<int> perm((size_t)ctx->Hc * ctx->Hr);
    for (int col = 0; col < ctx->Hc; ++col) {
      int base = col * ctx->Hr, len0 = ctx->mlen[2 * col], t = 0;
      for (int cl = 0; cl < 2; ++cl)
        for (int par = 0; par < 2; ++par)
          for (int k = 0; k < ctx->Hr; ++k)
            if ((k < len0 ? 0 : 1) == cl && ctx->hs[base + k] == par) perm[(size_t)col * ctx->Hr + t++] = k;
    }
    TRY(dalloc(ctx, &ctx->d_aperm, perm.size())); TRY(upload(ctx, ctx->d_aperm, perm));
  }
  {  // solve blocks: one degree l, up to 16 orders m (all (l, m) share the factors of l)
    std::vector<int> bl, bnh;
    for (int l = 0; l < L; ++l) {
      std::vector<int> nhs;
      for (int mi = 0; mi < ctx->M; ++mi)
        if (lm2nh[(size_t)mi * L + l] >= 0) nhs.push_back(lm2nh[(size_t)mi * L + l]);
      for (size_t i0 = 0; i0 < nhs.size(); i0 += 16) {
        bl.push_back(l);
        for (size_t i = i0; i < i0 + 16; ++i) bnh.push_back(i < nhs.size() ? nhs[i] : -1);
      }
    }
    ctx->nsblk = (int)bl.size();
    TRY(dalloc(ctx, &ctx->d_sblk_l, bl.size())); TRY(upload(ctx, ctx->d_sblk_l, bl));
    TRY(dalloc(ctx, &ctx->d_sblk_nh, bnh.size())); TRY(upload(ctx, ctx->d_sblk_nh, bnh));
  }
  // FFT twiddles (long double host trigonometry, rounded once)
  {
    std::vector<double2> tw2(ctx->P2), twh(ctx->Ph);
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < ctx->P2; ++k) {
      long double a = 2.0L * PI * (long double)k / (long double)ctx->P2;
      tw2[k] = make_double2((double)cosl(a), (double)sinl(a));
    }
    for (int k = 0; k < ctx->Ph; ++k) {
      long double a = 2.0L * PI * (long double)k / (long double)ctx->Ph;
      twh[k] = make_double2((double)cosl(a), (double)sinl(a));
    }
    TRY(dalloc(ctx, &ctx->d_tw2, tw2.size())); TRY(upload(ctx, ctx->d_tw2, tw2));
    TRY(dalloc(ctx, &ctx->d_twh, twh.size())); TRY(upload(ctx, ctx->d_twh, twh));
  }
  TRY(dalloc(ctx, &ctx->d_leg, (size_t)8 * H * Th2));
  TRY(dalloc(ctx, &ctx->d_gp, Th)); TRY(dalloc(ctx, &ctx->d_gw, Th));
  TRY(dalloc(ctx, &ctx->d_sn, Th)); TRY(dalloc(ctx, &ctx->d_sn1, Th));
  TRY(dalloc(ctx, &ctx->d_r, (size_t)7 * N));
  ctx->d_rinv = ctx->d_r + (size_t)2 * N;
  TRY(dalloc(ctx, &ctx->d_ones, N));
  TRY(upload(ctx, ctx->d_ones, std::vector<double>(N, 1.0)));
  TRY(dalloc(ctx, &ctx->d_dr, (size_t)KL * (2 * KL + 1) * N));
  TRY(dalloc(ctx, &ctx->d_r1dr, (size_t)(2 * KL + 1) * N));
  TRY(dalloc(ctx, &ctx->d_radlap, (size_t)(2 * KL + 1) * N));
  TRY(dalloc(ctx, &ctx->d_intr2dr, N));
  TRY(dalloc(ctx, &ctx->d_ref, (size_t)7 * N));
  TRY(dalloc(ctx, &ctx->d_laps, (size_t)LAP_NBAND * (2 * KL + 1) * N));
  TRY(dalloc(ctx, &ctx->d_compr1dr, (size_t)(2 * KL + 1) * N));
  TRY(dalloc(ctx, &ctx->d_wts, (size_t)4 * N));
  {  // reference state: Boussinesq rho = T = 0, eta = 1 (io.F90:545-556); anelastic until
     // lsd_set_reference_state: rho = T = eta = 1, gradients 0
    std::vector<double> ref((size_t)7 * N, 0.0);
    for (int n = 0; n < N; ++n) {
      ref[(size_t)REF_ETA * N + n] = 1.0;
      if (!c.boussinesq) { ref[(size_t)REF_RHO * N + n] = 1.0; ref[(size_t)REF_T * N + n] = 1.0; }
    }
    TRY(upload(ctx, ctx->d_ref, ref));
  }
  for (int nh = 0; nh < H; ++nh) {
    if (ctx->hl[nh] == 1 && ctx->hm[nh] == 0) ctx->nh_l1m0 = nh;
    if (ctx->hl[nh] == 1 && ctx->hm[nh] == 1) ctx->nh_l1m1 = nh;
  }
  const int NL = ctx->NL;
  const size_t lus = (size_t)OP_NFAM * L * NL * (3 * KL + 1);
  TRY(dalloc(ctx, &ctx->d_lu, lus)); TRY(dalloc(ctx, &ctx->d_lus, lus));
  TRY(dalloc(ctx, &ctx->d_y, (size_t)OP_NFAM * N * (2 * KL + 1) * L));
  TRY(dalloc(ctx, &ctx->d_yt, (size_t)OP_NFAM * N * (2 * KL + 1) * L));
  TRY(dalloc(ctx, &ctx->d_ipiv, (size_t)OP_NFAM * L * NL)); TRY(dalloc(ctx, &ctx->d_ipivs, (size_t)OP_NFAM * L * NL));
  if (ctx->Nic > 1) {  // the inner core's mesh, field, saved terms and Y bands
    const int Ni = ctx->Nic;
    TRY(dalloc(ctx, &ctx->d_icr, (size_t)7 * Ni));
    TRY(dalloc(ctx, &ctx->d_icdr, (size_t)KL * (2 * KL + 1) * Ni));
    TRY(dalloc(ctx, &ctx->d_icradlap, (size_t)(2 * KL + 1) * Ni));
    TRY(dalloc(ctx, &ctx->d_icr1dr, (size_t)(2 * KL + 1) * Ni));
    TRY(dalloc(ctx, &ctx->d_icintr2dr, Ni));
    TRY(dalloc(ctx, &ctx->d_icwts, (size_t)4 * Ni));
    TRY(dalloc(ctx, &ctx->d_iclaps, (size_t)LAP_NBAND * (2 * KL + 1) * Ni));
    TRY(dalloc(ctx, &ctx->d_iccompr1dr, (size_t)(2 * KL + 1) * Ni));
    TRY(dalloc(ctx, &ctx->d_icref, (size_t)7 * Ni));
    std::vector<double> ref((size_t)7 * Ni, 0.0);
    for (int n = 0; n < Ni; ++n) ref[(size_t)REF_ETA * Ni + n] = 1.0;
    TRY(upload(ctx, ctx->d_icref, ref));
    TRY(dalloc(ctx, &ctx->d_icyt, (size_t)2 * Ni * (2 * KL + 1) * L));
    TRY(dalloc(ctx, &ctx->d_icstate, (size_t)2 * Ni * H)); TRY(dalloc(ctx, &ctx->d_icsv, (size_t)2 * Ni * H));
    CTRY(cudaMemsetAsync(ctx->d_icstate, 0, sizeof(cplx) * 2 * Ni * H, ctx->stream));
    CTRY(cudaMemsetAsync(ctx->d_icsv, 0, sizeof(cplx) * 2 * Ni * H, ctx->stream));
  }
  TRY(dalloc(ctx, &ctx->d_rot, (size_t)ROT_NSLOT + 4 * ctx->HB));  // + the torque sums per half-row
  CTRY(cudaMemsetAsync(ctx->d_rot, 0, sizeof(double) * (ROT_NSLOT + 4 * ctx->HB), ctx->stream));
  TRY(dalloc(ctx, &ctx->d_gwP0, Th));
  {  // rot_precompute (rotation.F90:20-33): 8 pi / 15 r_i^5, r_i = rratio / (1 - rratio)
    const double ri = c.rratio / (1.0 - c.rratio), r2 = ri * ri, r4 = r2 * r2;
    ctx->rot_inertia = (8.0 * 3.1415926535897931 / 15.0) * (r4 * ri);
  }
  TRY(dalloc(ctx, &ctx->d_info, (size_t)OP_NFAM * L));
  TRY(dalloc(ctx, &ctx->d_gre, (size_t)L * 2 * N)); TRY(dalloc(ctx, &ctx->d_invg, (size_t)L * 4));
  TRY(dalloc(ctx, &ctx->d_gret, (size_t)L * 2 * N));
  TRY(dalloc(ctx, &ctx->d_grescr, (size_t)L * N));
  const size_t F = (size_t)N * H;
  TRY(dalloc(ctx, &ctx->d_state, LSD_NFIELD * F)); TRY(dalloc(ctx, &ctx->d_nl, LSD_NFIELD * F));
  TRY(dalloc(ctx, &ctx->d_sv, LSD_NFIELD * F));
  CTRY(cudaMemsetAsync(ctx->d_state, 0, sizeof(cplx) * LSD_NFIELD * F, ctx->stream));
  CTRY(cudaMemsetAsync(ctx->d_nl, 0, sizeof(cplx) * LSD_NFIELD * F, ctx->stream));
  CTRY(cudaMemsetAsync(ctx->d_sv, 0, sizeof(cplx) * LSD_NFIELD * F, ctx->stream));
  // 12 solve work columns / evaluation slots + dC + dComp (+ dr q, dr s, dr t, anelastic)
  ctx->nspec = c.boussinesq ? 14 : 17;
  TRY(dalloc(ctx, &ctx->d_spec, (size_t)ctx->nspec * F));
  // 15 synthesised fields (FFT layout) + 7 products (analysis layout); composition adds
  // grad Comp (3) and its product (1), the anelastic equations dr u (3)
  ctx->nfour = 22 + (c.comp_tstep ? 4 : 0) + (c.boussinesq ? 0 : 3);
  if (lsd_products_smem(ctx) > 224 * 1024) {
    int rc2 = lsd_fail(ctx, LSD_EARG, "the products' FFT rows of this field set do not fit in shared memory at this M");
    free_ctx(ctx);
    return rc2;
  }
  TRY(dalloc(ctx, &ctx->d_four, (size_t)ctx->nfour * N * ctx->HB * NM * 4));
  TRY(dalloc(ctx, &ctx->d_red, (size_t)128 + 48 * N));
  TRY(dalloc(ctx, &ctx->d_cpart, (size_t)8 * ((H + 31) / 32)));
  TRY(dalloc(ctx, &ctx->d_cfl, (size_t)2 * N + 1));
  CTRY(cudaMallocHost((void**)&ctx->h_red, sizeof(double) * 64));
  // pinned staging: three spectral fields, and at least the host staging of the energy
  // diagnostics ((75 + 2 KL) N + 6 doubles, lsd_energy_device / lsd_energy_static)
  ctx->h_pin_bytes = std::max(sizeof(cplx) * F * 3, sizeof(double) * ((size_t)(75 + 2 * c.KL) * N + 16));
  CTRY(cudaMallocHost((void**)&ctx->h_pin, ctx->h_pin_bytes));
  TRY(dalloc(ctx, &ctx->d_pc, 1));
  TRY(dalloc(ctx, &ctx->d_opfail, 1));
  CTRY(cudaMallocHost((void**)&ctx->h_pc, sizeof(PcDev)));
  CTRY(cudaMemsetAsync(ctx->d_pc, 0, sizeof(PcDev), ctx->stream));
  TRY(lsd_build_tables(ctx));
  TRY(lsd_build_operators(ctx));
  if (c.precision == LSD_PREC_OZAKI) TRY(lsd_ozaki_setup(ctx));
  if (c.autotune) TRY(lsd_autotune(ctx));
#undef TRY
#undef CTRY
  *out = ctx;
  return LSD_OK;
}

int lsd_set_reference_state(lsd_ctx* ctx, const double* prof) {
  if (!ctx || !prof) return LSD_EARG;
  if (ctx->cfg.boussinesq) return lsd_fail(ctx, LSD_EARG, "reference state: the context solves the Boussinesq equations");
  const int N = ctx->N;
  for (int n = 0; n < N; ++n)
    if (!(prof[(size_t)REF_RHO * N + n] > 0.0) || !(prof[(size_t)REF_T * N + n] > 0.0))
      return lsd_fail(ctx, LSD_EARG, "reference state: rho and T must be positive at every shell");
  CUDA_TRY(cudaSetDevice(ctx->dev));
  CUDA_TRY(cudaMemcpyAsync(ctx->d_ref, prof, sizeof(double) * 7 * N, cudaMemcpyHostToDevice, ctx->stream));
  int rc = lsd_build_radial(ctx);
  if (rc) return rc;
  rc = lsd_build_operators(ctx);
  if (rc) return rc;
  ctx->have_refstate = true;
  ctx->have_eval = false;
  return LSD_OK;
}

int lsd_destroy(lsd_ctx* ctx) {
  free_ctx(ctx);
  return LSD_OK;
}

const char* lsd_last_error(const lsd_ctx* ctx) { return ctx ? ctx->err.c_str() : t_create_err.c_str(); }

int lsd_get_sizes(const lsd_ctx* c, lsd_sizes* s) {
  if (!c || !s) return LSD_EARG;
  s->H = c->H; s->Th = c->Th; s->Th2 = c->Th2; s->Ph = c->Ph; s->Ma = c->Ma; s->Hc = c->Hc; s->Hr = c->Hr;
  s->N = c->N; s->L = c->L; s->M = c->M; s->Mp = c->Mp; s->KL = c->KL;
  return LSD_OK;
}

int lsd_harmonics(const lsd_ctx* c, int* l, int* m, int* s) {
  if (!c || !l || !m || !s) return LSD_EARG;
  for (int i = 0; i < c->H; ++i) { l[i] = c->hl[i]; m[i] = c->hm[i]; s[i] = c->hs[i]; }
  return LSD_OK;
}
int lsd_theta_map(const lsd_ctx* c, int* thm) {
  if (!c || !thm) return LSD_EARG;
  for (int i = 0; i < c->NM; ++i) thm[i] = c->thm[i];
  return LSD_OK;
}

static int d2h(lsd_ctx* ctx, void* dst, const void* src, size_t bytes) {
  CUDA_TRY(cudaSetDevice(ctx->dev));
  CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return LSD_OK;
}

int lsd_radial_grid(const lsd_ctx* c, double* r) {
  if (!c || !r) return LSD_EARG;
  return d2h(const_cast<lsd_ctx*>(c), r, c->d_r + (size_t)4 * c->N, sizeof(double) * c->N);
}
int lsd_radial_weights(const lsd_ctx* c, double* w) {
  if (!c || !w) return LSD_EARG;
  return d2h(const_cast<lsd_ctx*>(c), w, c->d_intr2dr, sizeof(double) * c->N);
}
int lsd_gauss(const lsd_ctx* c, double* gp, double* gw) {
  if (!c || !gp || !gw) return LSD_EARG;
  int rc = d2h(const_cast<lsd_ctx*>(c), gp, c->d_gp, sizeof(double) * c->Th);
  if (rc) return rc;
  return d2h(const_cast<lsd_ctx*>(c), gw, c->d_gw, sizeof(double) * c->Th);
}
int lsd_legendre_table(const lsd_ctx* c, int which, double* out) {
  if (!c || !out || which < 0 || which > 7) return LSD_EARG;
  size_t T = (size_t)c->H * c->Th2;
  return d2h(const_cast<lsd_ctx*>(c), out, c->d_leg + (size_t)which * T, sizeof(double) * T);
}

// coll fields cross the boundary in the reference's layout (Re, Im as (N, H) column-major
// arrays); they are copied as they are and transposed into [n][nh] on the device
// (lsd_coll_to_state / lsd_state_to_coll), with a scratch area of the spectral buffers.
// the inner core's field (Nic > 1): [Nic][H] on the device
static cplx* ic_field(lsd_ctx* ctx, int field) {
  if (ctx->Nic <= 1 || (field != LSD_MAG_IC_TOR && field != LSD_MAG_IC_POL)) return nullptr;
  return ctx->d_icstate + (size_t)(field - LSD_MAG_IC_TOR) * ctx->Nic * ctx->H;
}
// ---- staged uploads ---------------------------------------------------------------------
// Staging slots: the six outer-core fields, then the inner core's two (Nic rows each).
static const int STAGE_SLOTS = LSD_NFIELD + 2;
static int stage_setup(lsd_ctx* ctx) {
  if (ctx->d_stage) return LSD_OK;
  CUDA_TRY(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  for (int k = 0; k < 2; ++k) {
    CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_staged[k], cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_committed[k], cudaEventDisableTiming));
  }
  const size_t F = (size_t)ctx->N * ctx->H;
  CUDA_TRY(cudaMalloc(&ctx->d_stage, sizeof(double) * 2 * STAGE_SLOTS * 2 * F));
  return LSD_OK;
}
static double* stage_ptr(lsd_ctx* ctx, int set, int slot) {
  const size_t F = (size_t)ctx->N * ctx->H;
  return ctx->d_stage + ((size_t)set * STAGE_SLOTS + slot) * 2 * F;
}

int lsd_stage_coll(lsd_ctx* ctx, int field, const double* re, const double* im) {
  if (!ctx || !re || !im) return LSD_EARG;
  const bool ic = field == LSD_MAG_IC_TOR || field == LSD_MAG_IC_POL;
  if ((ic && ctx->Nic <= 1) || (!ic && (field < 0 || field >= LSD_NFIELD))) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc = stage_setup(ctx);
  if (rc) return rc;
  const int set = ctx->stage_set;
  if (ctx->stage_mask[set] == 0u)  // the set's buffers are free once its last commit has run
    CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_committed[set], 0));
  const size_t n = (size_t)(ic ? ctx->Nic : ctx->N) * ctx->H;
  double* dst = stage_ptr(ctx, set, field);
  CUDA_TRY(cudaMemcpyAsync(dst, re, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->copy_stream));
  CUDA_TRY(cudaMemcpyAsync(dst + n, im, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->copy_stream));
  ctx->stage_mask[set] |= 1u << field;
  return LSD_OK;
}

int lsd_commit_staged(lsd_ctx* ctx) {
  if (!ctx) return LSD_EARG;
  const int set = ctx->stage_set;
  if (!ctx->d_stage || ctx->stage_mask[set] == 0u)
    return lsd_fail(ctx, LSD_ESTATE, "lsd_commit_staged: no field staged since the last commit");
  CUDA_TRY(cudaSetDevice(ctx->dev));
  CUDA_TRY(cudaEventRecord(ctx->ev_staged[set], ctx->copy_stream));
  CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_staged[set], 0));
  const size_t F = (size_t)ctx->N * ctx->H;
  for (int f = 0; f < STAGE_SLOTS; ++f) {
    if (!(ctx->stage_mask[set] & (1u << f))) continue;
    const bool ic = f >= LSD_NFIELD;
    const int rows = ic ? ctx->Nic : ctx->N;
    const size_t n = (size_t)rows * ctx->H;
    const double* src = stage_ptr(ctx, set, f);
    cplx* out = ic ? ctx->d_icstate + (size_t)(f - LSD_MAG_IC_TOR) * ctx->Nic * ctx->H : ctx->d_state + f * F;
    int rc = lsd_coll_to_state_n(ctx, rows, src, src + n, out);
    if (rc) return rc;
  }
  CUDA_TRY(cudaEventRecord(ctx->ev_committed[set], ctx->stream));
  ctx->stage_mask[set] = 0u;
  ctx->stage_set = 1 - set;
  ctx->have_eval = false;
  return LSD_OK;
}

int lsd_set_coll(lsd_ctx* ctx, int field, const double* re, const double* im) {
  if (!ctx || !re || !im) return LSD_EARG;
  if (cplx* ic = ic_field(ctx, field)) {
    CUDA_TRY(cudaSetDevice(ctx->dev));
    const size_t Fi = (size_t)ctx->Nic * ctx->H;
    double* stage = (double*)ctx->d_spec;
    CUDA_TRY(cudaMemcpyAsync(stage, re, sizeof(double) * Fi, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(stage + Fi, im, sizeof(double) * Fi, cudaMemcpyHostToDevice, ctx->stream));
    int rc = lsd_coll_to_state_n(ctx, ctx->Nic, stage, stage + Fi, ic);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->have_eval = false;
    return LSD_OK;
  }
  if (field < 0 || field >= LSD_NFIELD) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  const size_t F = (size_t)ctx->N * ctx->H;
  double* stage = (double*)ctx->d_spec;  // 2 F doubles: Re then Im
  CUDA_TRY(cudaMemcpyAsync(stage, re, sizeof(double) * F, cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaMemcpyAsync(stage + F, im, sizeof(double) * F, cudaMemcpyHostToDevice, ctx->stream));
  int rc = lsd_coll_to_state(ctx, stage, stage + F, ctx->d_state + field * F);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->have_eval = false;
  return LSD_OK;
}
static int coll_out(lsd_ctx* ctx, const cplx* src, double* re, double* im) {
  CUDA_TRY(cudaSetDevice(ctx->dev));
  const size_t F = (size_t)ctx->N * ctx->H;
  double* stage = (double*)ctx->d_spec;
  int rc = lsd_state_to_coll(ctx, src, stage, stage + F);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(re, stage, sizeof(double) * F, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaMemcpyAsync(im, stage + F, sizeof(double) * F, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return LSD_OK;
}
int lsd_get_coll(lsd_ctx* ctx, int field, double* re, double* im) {
  if (!ctx || !re || !im) return LSD_EARG;
  if (cplx* ic = ic_field(ctx, field)) {
    CUDA_TRY(cudaSetDevice(ctx->dev));
    const size_t Fi = (size_t)ctx->Nic * ctx->H;
    double* stage = (double*)ctx->d_spec;
    int rc = lsd_state_to_coll_n(ctx, ctx->Nic, ic, stage, stage + Fi);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(re, stage, sizeof(double) * Fi, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(im, stage + Fi, sizeof(double) * Fi, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return LSD_OK;
  }
  if (field < 0 || field >= LSD_NFIELD) return LSD_EARG;
  return coll_out(ctx, ctx->d_state + field * (size_t)ctx->N * ctx->H, re, im);
}
int lsd_get_nonlinear(lsd_ctx* ctx, int which, double* re, double* im) {
  if (!ctx || !re || !im || which < 0 || which >= LSD_NFIELD) return LSD_EARG;
  return coll_out(ctx, ctx->d_nl + which * (size_t)ctx->N * ctx->H, re, im);
}

int lsd_set_time(lsd_ctx* ctx, double t, double dt) {
  if (!ctx || !(dt > 0.0)) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  ctx->t = t;
  if (dt != ctx->dt) {
    ctx->dt = dt;
    int rc = lsd_build_operators(ctx);
    if (rc) return rc;
  }
  return LSD_OK;
}
// rot_omega (the state file's 'omega'); the rate at the last evaluation follows it
int lsd_set_rotation(lsd_ctx* ctx, double omega) {
  if (!ctx) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  const double w[2] = {omega, omega};
  CUDA_TRY(cudaMemcpyAsync(ctx->d_rot + ROT_OMEGA, w, sizeof(w), cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return LSD_OK;
}
int lsd_get_rotation(const lsd_ctx* cctx, double* out) {
  if (!cctx || !out) return LSD_EARG;
  lsd_ctx* ctx = const_cast<lsd_ctx*>(cctx);
  CUDA_TRY(cudaSetDevice(ctx->dev));
  double r[ROT_NSLOT];
  CUDA_TRY(cudaMemcpyAsync(r, ctx->d_rot, sizeof(r), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  out[0] = r[ROT_OMEGA]; out[1] = r[ROT_VEL]; out[2] = r[ROT_MAG];
  return LSD_OK;
}
// tim_dt, tim_corr_dt, tim_cfl_dt (the columns of io_write_timestep, io.F90:2343-2346)
int lsd_get_dt_control(const lsd_ctx* ctx, double* out) {
  if (!ctx || !out) return LSD_EARG;
  out[0] = ctx->dt; out[1] = ctx->corr_dt; out[2] = ctx->cfl_dt;
  return LSD_OK;
}
int lsd_get_time(const lsd_ctx* ctx, double* t, double* dt, int* step) {
  if (!ctx) return LSD_EARG;
  if (t) *t = ctx->t;
  if (dt) *dt = ctx->dt;
  if (step) *step = ctx->step;
  return LSD_OK;
}

// ---- host-buffer transforms ------------------------------------------------------------
static int spec_in(lsd_ctx* ctx, int slot, const double* re, const double* im) {
  const size_t F = (size_t)ctx->N * ctx->H;
  double* buf = ctx->h_pin + (size_t)slot * 2 * F;
  pack_spec(ctx, re, im, buf);
  CUDA_TRY(cudaMemcpyAsync(ctx->d_spec + slot * F, buf, sizeof(cplx) * F, cudaMemcpyHostToDevice, ctx->stream));
  return LSD_OK;
}
static int spec_out(lsd_ctx* ctx, int slot, double* re, double* im) {
  const size_t F = (size_t)ctx->N * ctx->H;
  double* buf = ctx->h_pin + (size_t)slot * 2 * F;
  CUDA_TRY(cudaMemcpyAsync(buf, ctx->d_spec + slot * F, sizeof(cplx) * F, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  unpack_spec(ctx, buf, re, im);
  return LSD_OK;
}
static size_t phys_count(const lsd_ctx* c) { return (size_t)c->N * c->Ph * c->Th; }

int lsd_tra_spec2phys(lsd_ctx* ctx, const double* s_re, const double* s_im, double* p) {
  if (!ctx || !s_re || !s_im || !p) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc;
  if ((rc = ensure_phys(ctx, 3))) return rc;
  if ((rc = spec_in(ctx, 0, s_re, s_im))) return rc;
  const size_t F = (size_t)ctx->N * ctx->H;
  (void)F;
  SynthGroup g;
  g.kind = SK_SCALAR;
  g.in[0] = ctx->d_spec; g.in[1] = g.in[2] = nullptr;
  g.out[0] = ctx->d_four; g.out[1] = g.out[2] = nullptr;
  if ((rc = time_begin(ctx))) return rc;
  if ((rc = lsd_launch_synth(ctx, &g, 1))) return rc;
  if ((rc = lsd_launch_c2r(ctx, ctx->d_four, ctx->d_phys, 1))) return rc;
  if ((rc = time_end(ctx))) return rc;
  if ((rc = d2h(ctx, p, ctx->d_phys, sizeof(double) * phys_count(ctx)))) return rc;
  return LSD_OK;
}

int lsd_tra_phys2spec(lsd_ctx* ctx, const double* p, double* s_re, double* s_im) {
  if (!ctx || !s_re || !s_im || !p) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc;
  if ((rc = ensure_phys(ctx, 3))) return rc;
  if ((rc = h2d(ctx, ctx->d_phys, p, sizeof(double) * phys_count(ctx)))) return rc;
  AnalGroup g;
  g.kind = AK_SCALAR;
  g.in[0] = ctx->d_four; g.in[1] = g.in[2] = nullptr;
  g.out[0] = ctx->d_spec; g.out[1] = g.out[2] = nullptr;
  if ((rc = time_begin(ctx))) return rc;
  if ((rc = lsd_launch_r2c(ctx, ctx->d_phys, ctx->d_four, 1))) return rc;
  if ((rc = lsd_launch_anal(ctx, &g, 1))) return rc;
  if ((rc = time_end(ctx))) return rc;
  return spec_out(ctx, 0, s_re, s_im);
}

int lsd_tra_qst2rtp(lsd_ctx* ctx, const double* q_re, const double* q_im, const double* s_re, const double* s_im,
                    const double* t_re, const double* t_im, double* r, double* th, double* ph) {
  if (!ctx || !q_re || !q_im || !s_re || !s_im || !t_re || !t_im || !r || !th || !ph) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc;
  if ((rc = ensure_phys(ctx, 3))) return rc;
  if ((rc = spec_in(ctx, 0, q_re, q_im)) || (rc = spec_in(ctx, 1, s_re, s_im)) || (rc = spec_in(ctx, 2, t_re, t_im))) return rc;
  const size_t F = (size_t)ctx->N * ctx->H, FF = (size_t)ctx->N * ctx->HB * ctx->NM * 4;
  SynthGroup g;
  g.kind = SK_VECTOR;
  for (int k = 0; k < 3; ++k) { g.in[k] = ctx->d_spec + k * F; g.out[k] = ctx->d_four + k * FF; }
  if ((rc = time_begin(ctx))) return rc;
  if ((rc = lsd_launch_synth(ctx, &g, 1))) return rc;
  if ((rc = lsd_launch_c2r(ctx, ctx->d_four, ctx->d_phys, 3))) return rc;
  if ((rc = time_end(ctx))) return rc;
  size_t P = phys_count(ctx);
  if ((rc = d2h(ctx, r, ctx->d_phys, sizeof(double) * P))) return rc;
  if ((rc = d2h(ctx, th, ctx->d_phys + P, sizeof(double) * P))) return rc;
  if ((rc = d2h(ctx, ph, ctx->d_phys + 2 * P, sizeof(double) * P))) return rc;
  return LSD_OK;
}

int lsd_tra_rtp2qst(lsd_ctx* ctx, const double* r, const double* th, const double* ph, double* q_re, double* q_im,
                    double* s_re, double* s_im, double* t_re, double* t_im) {
  if (!ctx || !q_re || !q_im || !s_re || !s_im || !t_re || !t_im || !r || !th || !ph) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc;
  if ((rc = ensure_phys(ctx, 3))) return rc;
  size_t P = phys_count(ctx);
  if ((rc = h2d(ctx, ctx->d_phys, r, sizeof(double) * P))) return rc;
  if ((rc = h2d(ctx, ctx->d_phys + P, th, sizeof(double) * P))) return rc;
  if ((rc = h2d(ctx, ctx->d_phys + 2 * P, ph, sizeof(double) * P))) return rc;
  const size_t F = (size_t)ctx->N * ctx->H, FF = (size_t)ctx->N * ctx->HB * ctx->NM * 4;
  AnalGroup g;
  g.kind = AK_VECTOR;
  for (int k = 0; k < 3; ++k) { g.in[k] = ctx->d_four + k * FF; g.out[k] = ctx->d_spec + k * F; }
  if ((rc = time_begin(ctx))) return rc;
  if ((rc = lsd_launch_r2c(ctx, ctx->d_phys, ctx->d_four, 3))) return rc;
  if ((rc = lsd_launch_anal(ctx, &g, 1))) return rc;
  if ((rc = time_end(ctx))) return rc;
  if ((rc = spec_out(ctx, 0, q_re, q_im)) || (rc = spec_out(ctx, 1, s_re, s_im)) || (rc = spec_out(ctx, 2, t_re, t_im))) return rc;
  return LSD_OK;
}

int lsd_tra_grad(lsd_ctx* ctx, const double* s_re, const double* s_im, double* th, double* ph) {
  if (!ctx || !s_re || !s_im || !th || !ph) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc;
  if ((rc = ensure_phys(ctx, 3))) return rc;
  if ((rc = spec_in(ctx, 0, s_re, s_im))) return rc;
  const size_t FF = (size_t)ctx->N * ctx->HB * ctx->NM * 4;
  SynthGroup g;
  g.kind = SK_GRAD2;
  g.in[0] = ctx->d_spec; g.in[1] = g.in[2] = nullptr;
  g.out[0] = ctx->d_four; g.out[1] = ctx->d_four + FF; g.out[2] = nullptr;
  if ((rc = time_begin(ctx))) return rc;
  if ((rc = lsd_launch_synth(ctx, &g, 1))) return rc;
  if ((rc = lsd_launch_c2r(ctx, ctx->d_four, ctx->d_phys, 2))) return rc;
  if ((rc = time_end(ctx))) return rc;
  size_t P = phys_count(ctx);
  if ((rc = d2h(ctx, th, ctx->d_phys, sizeof(double) * P))) return rc;
  if ((rc = d2h(ctx, ph, ctx->d_phys + P, sizeof(double) * P))) return rc;
  return LSD_OK;
}

// tra_dth (transform.fftw3.F90:1006-1031): the theta part of tra_grad without the 1/r
int lsd_tra_dth(lsd_ctx* ctx, const double* s_re, const double* s_im, double* p) {
  if (!ctx || !s_re || !s_im || !p) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc;
  if ((rc = ensure_phys(ctx, 3))) return rc;
  if ((rc = spec_in(ctx, 0, s_re, s_im))) return rc;
  const size_t FF = (size_t)ctx->N * ctx->HB * ctx->NM * 4;
  SynthGroup g;
  g.kind = SK_GRAD2;
  g.in[0] = ctx->d_spec; g.in[1] = g.in[2] = nullptr;
  g.out[0] = ctx->d_four; g.out[1] = ctx->d_four + FF; g.out[2] = nullptr;
  if ((rc = time_begin(ctx))) return rc;
  ctx->d_rinv = ctx->d_ones;  // c * 1.0 == c: the sums of tra_dth
  rc = lsd_launch_synth(ctx, &g, 1);
  ctx->d_rinv = ctx->d_r + (size_t)2 * ctx->N;
  if (rc) return rc;
  if ((rc = lsd_launch_c2r(ctx, ctx->d_four, ctx->d_phys, 1))) return rc;
  if ((rc = time_end(ctx))) return rc;
  if ((rc = d2h(ctx, p, ctx->d_phys, sizeof(double) * phys_count(ctx)))) return rc;
  return LSD_OK;
}

// tra_qst2rtp_vel (transform.fftw3.F90:611-714): two vector syntheses, (q, s, t) and
// (dq, ds, dt), and qv1 / qv2 formed from the u_th, u_ph theta-Fourier rows.
int lsd_tra_qst2rtp_vel(lsd_ctx* ctx, const double* q_re, const double* q_im, const double* s_re,
                        const double* s_im, const double* t_re, const double* t_im, const double* qr_re,
                        const double* qr_im, const double* sr_re, const double* sr_im, const double* tr_re,
                        const double* tr_im, double* r, double* th, double* ph, double* dur, double* qv1,
                        double* dutr, double* dupr, double* qv2) {
  const double* in[12] = {q_re, q_im, s_re, s_im, t_re, t_im, qr_re, qr_im, sr_re, sr_im, tr_re, tr_im};
  double* out[8] = {r, th, ph, dur, qv1, dutr, dupr, qv2};
  if (!ctx) return LSD_EARG;
  for (const double* p : in) if (!p) return LSD_EARG;
  for (double* p : out) if (!p) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc;
  if ((rc = ensure_phys(ctx, 8))) return rc;
  const size_t F = (size_t)ctx->N * ctx->H, FF = (size_t)ctx->N * ctx->HB * ctx->NM * 4;
  for (int k = 0; k < 6; ++k) {  // one pinned slot, reused: upload field by field
    if ((rc = spec_in(ctx, 0, in[2 * k], in[2 * k + 1]))) return rc;
    CUDA_TRY(cudaMemcpyAsync(ctx->d_spec + (size_t)(6 + k) * F, ctx->d_spec, sizeof(cplx) * F,
                             cudaMemcpyDeviceToDevice, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  }
  cplx* fo = ctx->d_four;
  SynthGroup g[2];
  const int slots[2][3] = {{0, 1, 2}, {3, 5, 6}};  // r th ph ; dur dutr dupr
  for (int i = 0; i < 2; ++i) {
    g[i].kind = SK_VECTOR;
    for (int k = 0; k < 3; ++k) { g[i].in[k] = ctx->d_spec + (size_t)(6 + 3 * i + k) * F; g[i].out[k] = fo + slots[i][k] * FF; }
  }
  if ((rc = time_begin(ctx))) return rc;
  if ((rc = lsd_launch_synth(ctx, g, 2))) return rc;
  if ((rc = lsd_launch_qv(ctx, fo + 1 * FF, fo + 2 * FF, fo + 4 * FF, fo + 7 * FF))) return rc;
  if ((rc = lsd_launch_c2r(ctx, fo, ctx->d_phys, 8))) return rc;
  if ((rc = time_end(ctx))) return rc;
  size_t P = phys_count(ctx);
  for (int k = 0; k < 8; ++k)
    if ((rc = d2h(ctx, out[k], ctx->d_phys + k * P, sizeof(double) * P))) return rc;
  return LSD_OK;
}

// ---- device-resident batched transforms --------------------------------------------------
int lsd_sht_synth_device(lsd_ctx* ctx, int nbatch, const double* d_spec, double* d_phys) {
  if (!ctx || !d_spec || !d_phys || nbatch < 1) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  const size_t F = (size_t)ctx->N * ctx->H, FF = (size_t)ctx->N * ctx->HB * ctx->NM * 4, P = phys_count(ctx);
  const cplx* in = (const cplx*)d_spec;
  for (int b0 = 0; b0 < nbatch; b0 += ctx->nfour) {
    int nb = std::min(ctx->nfour, nbatch - b0);
    for (int g0 = 0; g0 < nb; g0 += 6) {
      SynthGroup g[6];
      int ng = std::min(6, nb - g0);
      for (int i = 0; i < ng; ++i) {
        g[i].kind = SK_SCALAR;
        g[i].in[0] = in + (size_t)(b0 + g0 + i) * F; g[i].in[1] = g[i].in[2] = nullptr;
        g[i].out[0] = ctx->d_four + (size_t)(g0 + i) * FF; g[i].out[1] = g[i].out[2] = nullptr;
      }
      int rc = lsd_launch_synth(ctx, g, ng);
      if (rc) return rc;
    }
    int rc = lsd_launch_c2r(ctx, ctx->d_four, d_phys + (size_t)b0 * P, nb);
    if (rc) return rc;
  }
  return LSD_OK;
}

int lsd_sht_analys_device(lsd_ctx* ctx, int nbatch, const double* d_phys, double* d_spec) {
  if (!ctx || !d_spec || !d_phys || nbatch < 1) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  const size_t F = (size_t)ctx->N * ctx->H, FF = (size_t)ctx->N * ctx->HB * ctx->NM * 4, P = phys_count(ctx);
  cplx* out = (cplx*)d_spec;
  for (int b0 = 0; b0 < nbatch; b0 += ctx->nfour) {
    int nb = std::min(ctx->nfour, nbatch - b0);
    int rc = lsd_launch_r2c(ctx, d_phys + (size_t)b0 * P, ctx->d_four, nb);
    if (rc) return rc;
    for (int g0 = 0; g0 < nb; g0 += 4) {
      AnalGroup g[4];
      int ng = std::min(4, nb - g0);
      for (int i = 0; i < ng; ++i) {
        g[i].kind = AK_SCALAR;
        g[i].in[0] = ctx->d_four + (size_t)(g0 + i) * FF; g[i].in[1] = g[i].in[2] = nullptr;
        g[i].out[0] = out + (size_t)(b0 + g0 + i) * F; g[i].out[1] = g[i].out[2] = nullptr;
      }
      rc = lsd_launch_anal(ctx, g, ng);
      if (rc) return rc;
    }
  }
  return LSD_OK;
}

// ---- time stepping ---------------------------------------------------------------------
int lsd_matrices(lsd_ctx* ctx) {
  if (!ctx) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  return lsd_build_operators(ctx);
}

int lsd_nonlinear(lsd_ctx* ctx) {
  if (!ctx) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc;
  if ((rc = time_begin(ctx))) return rc;
  if ((rc = lsd_eval(ctx))) return rc;
  if ((rc = time_end(ctx))) return rc;
  ctx->have_eval = true;
  return LSD_OK;
}

int lsd_predictor(lsd_ctx* ctx) {
  if (!ctx) return LSD_EARG;
  if (!ctx->have_eval) return lsd_fail(ctx, LSD_ESTATE, "predictor needs a nonlinear evaluation first");
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc = lsd_pred(ctx);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->it = 1;
  ctx->have_eval = false;
  return LSD_OK;
}

int lsd_corrector(lsd_ctx* ctx, double* dterr) {
  if (!ctx) return LSD_EARG;
  if (!ctx->have_eval || ctx->it == 0) return lsd_fail(ctx, LSD_ESTATE, "corrector needs a predictor and an evaluation");
  CUDA_TRY(cudaSetDevice(ctx->dev));
  ctx->dterr = 0.0;
  int rc = lsd_corr(ctx);
  if (!rc) rc = finish_corrector(ctx);
  if (rc) return rc;
  if (dterr) *dterr = ctx->dterr;
  ctx->have_eval = false;
  return LSD_OK;
}

int lsd_step(lsd_ctx* ctx, int nsteps, lsd_stats* stats) {
  if (!ctx || nsteps < 0) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  int rc;
  int done = 0, corr = 0, evals = 0;
  long long kernels = 0;
  double last = 0.0;
  const long long l0 = ctx->launches;
  if ((rc = time_begin(ctx))) return rc;
  if (ctx->it != 0 && nsteps > 0) {
    if ((rc = finish_open_step(ctx, &corr, &evals, &last))) return rc;
    ++done;
    kernels += ctx->launches - l0;
  }
  if (done < nsteps) {
    if ((rc = step_graph_enqueue(ctx, nsteps - done))) return rc;
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    rc = step_graph_finish(ctx, &done, &corr, &evals, &last, &kernels);
    ctx->launches = l0 + kernels;
    if (rc) return rc;
  }
  if ((rc = time_end(ctx))) return rc;
  ctx->have_eval = false;
  if (stats) {
    stats->steps_done = done; stats->correctors = corr; stats->evaluations = evals;
    stats->kernel_launches = (int)(ctx->launches - l0); stats->last_dterr = last;
    stats->t = ctx->t; stats->dt = ctx->dt;
  }
  return LSD_OK;
}

// ---- ensembles: independent runs stepped together ---------------------------------------
// One graph holds every member's step loop (the one-graph step of lsd_step, all nsteps,
// no host decision inside) as a branch of its own, forked from and joined to the
// ensemble's stream: lsd_ensemble_step is one graph launch for all members, whose kernels
// run concurrently as the graph's independent branches.
struct lsd_ensemble {
  std::vector<lsd_ctx*> m;
  std::string err;
  cudaStream_t stream = nullptr;          // the stream the ensemble's graph runs on
  cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> join;          // one per member
  cudaGraphExec_t g = nullptr;
  float last_ms = 0.f;
};

namespace {
void ensemble_free(lsd_ensemble* e) {
  if (!e) return;
  if (!e->m.empty()) cudaSetDevice(e->m[0]->dev);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->g) cudaGraphExecDestroy(e->g);
  for (cudaEvent_t ev : e->join)
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : {e->fork, e->ev0, e->ev1})
    if (ev) cudaEventDestroy(ev);
  if (e->stream) cudaStreamDestroy(e->stream);
  for (lsd_ctx* c : e->m) lsd_destroy(c);
  delete e;
}

// the ensemble's graph: fork to every member's stream, each member's step loop, join
int ensemble_capture(lsd_ensemble* e) {
  const int n = (int)e->m.size();
  if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    e->err = "ensemble graph: begin capture";
    return LSD_ECUDA;
  }
  int rc = LSD_OK;
  cudaError_t ce = cudaEventRecord(e->fork, e->stream);
  for (int i = 0; i < n && !rc && ce == cudaSuccess; ++i) {
    lsd_ctx* c = e->m[i];
    ce = cudaStreamWaitEvent(c->stream, e->fork, 0);
    if (ce == cudaSuccess) rc = capture_step_into(c);
    if (rc) { e->err = "member " + std::to_string(i) + ": " + c->err; break; }
    if (ce == cudaSuccess) ce = cudaEventRecord(e->join[i], c->stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->stream, e->join[i], 0);
  }
  cudaGraph_t g = nullptr;
  cudaError_t ee = cudaStreamEndCapture(e->stream, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (ce != cudaSuccess || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    e->err = std::string("ensemble graph capture: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ee);
    return LSD_ECUDA;
  }
  cudaError_t ie = cudaGraphInstantiate(&e->g, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) {
    e->err = std::string("ensemble graph instantiate: ") + cudaGetErrorString(ie);
    return LSD_ECUDA;
  }
  return LSD_OK;
}
}  // namespace

int lsd_ensemble_create(int n, const lsd_config* cfgs, lsd_ensemble** out) {
  if (!cfgs || !out || n < 1) return LSD_EARG;
  *out = nullptr;
  lsd_ensemble* e = new (std::nothrow) lsd_ensemble();
  if (!e) return LSD_ENOMEM;
  for (int i = 0; i < n; ++i) {
    lsd_ctx* c = nullptr;
    int rc = lsd_create(&cfgs[i], &c);
    if (rc) {
      for (lsd_ctx* x : e->m) lsd_destroy(x);
      delete e;
      return rc;
    }
    if (i > 0 && c->dev != e->m[0]->dev) {
      lsd_destroy(c);
      for (lsd_ctx* x : e->m) lsd_destroy(x);
      delete e;
      return LSD_EARG;
    }
    e->m.push_back(c);
  }
  cudaSetDevice(e->m[0]->dev);
  bool ok = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaEventCreate(&e->ev0) == cudaSuccess && cudaEventCreate(&e->ev1) == cudaSuccess;
  e->join.assign(n, nullptr);
  for (int i = 0; i < n && ok; ++i) ok = cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    ensemble_free(e);
    return LSD_ECUDA;
  }
  *out = e;
  return LSD_OK;
}

int lsd_ensemble_destroy(lsd_ensemble* e) {
  ensemble_free(e);
  return LSD_OK;
}

int lsd_ensemble_size(const lsd_ensemble* e) { return e ? (int)e->m.size() : 0; }

int lsd_ensemble_member(lsd_ensemble* e, int i, lsd_ctx** ctx) {
  if (!e || !ctx || i < 0 || i >= (int)e->m.size()) return LSD_EARG;
  *ctx = e->m[i];
  return LSD_OK;
}

const char* lsd_ensemble_last_error(const lsd_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }

int lsd_ensemble_step(lsd_ensemble* e, int nsteps, lsd_stats* stats) {
  if (!e || nsteps < 0) return LSD_EARG;
  const int n = (int)e->m.size();
  auto fail = [&](int i, int rc) {
    e->err = "member " + std::to_string(i) + ": " + e->m[i]->err;
    return rc;
  };
  if (cudaSetDevice(e->m[0]->dev) != cudaSuccess) return LSD_ECUDA;
  std::vector<int> done(n, 0), corr(n, 0), evals(n, 0);
  std::vector<long long> l0(n), kernels(n, 0);
  std::vector<double> last(n, 0.0);
  bool any = false;
  for (int i = 0; i < n; ++i) {  // steps begun by single predictor / corrector calls
    lsd_ctx* c = e->m[i];
    l0[i] = c->launches;
    if (c->it != 0 && nsteps > 0) {
      int rc = finish_open_step(c, &corr[i], &evals[i], &last[i]);
      if (rc) return fail(i, rc);
      ++done[i];
      kernels[i] += c->launches - l0[i];
    }
    any = any || done[i] < nsteps;
  }
  if (any) {
    if (!e->g) {
      int rc = ensemble_capture(e);
      if (rc) return rc;
    }
    // the members' queued work first (their own streams), then the graph on the ensemble's
    cudaError_t ce = cudaSuccess;
    for (int i = 0; i < n && ce == cudaSuccess; ++i) {
      ce = cudaEventRecord(e->join[i], e->m[i]->stream);
      if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->stream, e->join[i], 0);
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(e->ev0, e->stream);
    for (int i = 0; i < n; ++i) {
      int rc = pc_upload(e->m[i], nsteps - done[i], e->stream);
      if (rc) return fail(i, rc);
    }
    if (ce == cudaSuccess) ce = cudaGraphLaunch(e->g, e->stream);
    for (int i = 0; i < n; ++i) {
      int rc = pc_download(e->m[i], e->stream);
      if (rc) return fail(i, rc);
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(e->ev1, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&e->last_ms, e->ev0, e->ev1);
    if (ce != cudaSuccess) {
      e->err = std::string("ensemble graph launch: ") + cudaGetErrorString(ce);
      return LSD_ECUDA;
    }
  }
  for (int i = 0; i < n; ++i) {
    lsd_ctx* c = e->m[i];
    if (done[i] < nsteps) {
      int rc = step_graph_finish(c, &done[i], &corr[i], &evals[i], &last[i], &kernels[i]);
      c->launches = l0[i] + kernels[i];
      if (rc) return fail(i, rc);
    }
    if (c->oz) {
      int rc = lsd_ozaki_check(c);
      if (rc) return fail(i, rc);
    }
    c->last_ms = e->last_ms;
    c->have_eval = false;
    if (stats) {
      stats[i].steps_done = done[i]; stats[i].correctors = corr[i]; stats[i].evaluations = evals[i];
      stats[i].kernel_launches = (int)(c->launches - l0[i]); stats[i].last_dterr = last[i];
      stats[i].t = c->t; stats[i].dt = c->dt;
    }
  }
  return LSD_OK;
}

int lsd_ensemble_last_elapsed_ms(const lsd_ensemble* e, double* ms) {
  if (!e || !ms) return LSD_EARG;
  *ms = e->last_ms;
  return LSD_OK;
}

int lsd_get_stream(const lsd_ctx* ctx, void** stream) {
  if (!ctx || !stream) return LSD_EARG;
  *stream = (void*)ctx->stream;
  return LSD_OK;
}

int lsd_tim_check_cgce(const lsd_config* cfg, lsd_pc_state* s) {
  if (!cfg || !s) return LSD_EARG;
  PcState st;
  std::memcpy(&st, s, sizeof(st));
  const bool ok = pc_check_cgce(st, pc_params(*cfg));
  std::memcpy(s, &st, sizeof(st));
  return ok ? LSD_OK : LSD_ENOTCONVERGED;
}

int lsd_tim_new_tstep(const lsd_config* cfg, lsd_pc_state* s, int* new_dt) {
  if (!cfg || !s) return LSD_EARG;
  PcState st;
  std::memcpy(&st, s, sizeof(st));
  const bool nd = pc_new_tstep(st, pc_params(*cfg));
  std::memcpy(s, &st, sizeof(st));
  if (new_dt) *new_dt = nd ? 1 : 0;
  return LSD_OK;
}

int lsd_energies(lsd_ctx* ctx, double* out) {
  if (!ctx || !out) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  return lsd_energy_device(ctx, out);
}

int lsd_diagnostics(lsd_ctx* ctx, double* scalars, double* spectra, double* profiles) {
  if (!ctx || !scalars) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  return lsd_diagnostics_device(ctx, scalars, spectra, profiles);
}

int lsd_energies_static(lsd_ctx* ctx, double* out) {
  if (!ctx || !out) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  return lsd_energy_static(ctx, out);
}

int lsd_banded_factor_device(lsd_ctx* ctx, int n, int kl, int nmat, double* d_ab, int* d_ipiv, int* d_info) {
  if (!ctx || n < 1 || kl < 1 || kl > LSD_MAX_KL || nmat < 1 || !d_ab || !d_ipiv || !d_info) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  return lsd_factor_batch(ctx, n, kl, nmat, d_ab, d_ipiv, d_info);
}
int lsd_banded_solve_device(lsd_ctx* ctx, int n, int kl, int nmat, const double* d_ab, const int* d_ipiv, int nrhs,
                            const int* d_map, double* d_b) {
  if (!ctx || n < 1 || kl < 1 || kl > LSD_MAX_KL || nmat < 1 || nrhs < 1 || !d_ab || !d_ipiv || !d_map || !d_b) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  return lsd_solve_batch(ctx, n, kl, nmat, d_ab, d_ipiv, nrhs, d_map, d_b);
}

int lsd_operator_solve_device(lsd_ctx* ctx, int nfield, const int* fields, double* d_data) {
  if (!ctx || !fields || !d_data) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  return lsd_operator_solve(ctx, nfield, fields, d_data);
}

int lsd_profile_phases(lsd_ctx* ctx, double* ms, int* nphase) {
  if (!ctx || !ms || !nphase || *nphase < LSD_NPHASE) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  // ev[0] start, ev[1..5] after the five evaluation phases, ev[6] after the predictor,
  // ev[7], ev[8] around the corrector solve of the second evaluation
  cudaEvent_t ev[9];
  for (int i = 0; i < 9; ++i) CUDA_TRY(cudaEventCreate(&ev[i]));
  CUDA_TRY(cudaEventRecord(ev[0], ctx->stream));
  int rc = lsd_eval_marked(ctx, ev + 1);
  if (!rc) rc = lsd_pred(ctx);
  if (!rc) { cudaEventRecord(ev[6], ctx->stream); rc = lsd_eval(ctx); }
  if (!rc) { cudaEventRecord(ev[7], ctx->stream); rc = lsd_corr(ctx); }
  if (!rc) cudaEventRecord(ev[8], ctx->stream);
  if (!rc) rc = finish_corrector(ctx);
  if (!rc) {
    float t = 0.f;
    for (int i = 0; i < 6; ++i) {
      cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
      ms[i] = t;
    }
    cudaEventElapsedTime(&t, ev[7], ev[8]);
    ms[6] = t;
    *nphase = LSD_NPHASE;
  }
  for (int i = 0; i < 9; ++i) cudaEventDestroy(ev[i]);
  ctx->it = 0;
  ctx->dterr = 0.0;
  ctx->have_eval = false;
  ctx->t = ctx->t + ctx->dt;
  ctx->step = ctx->step + 1;
  return rc;
}

int lsd_synchronize(lsd_ctx* ctx) {
  if (!ctx) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (ctx->copy_stream) CUDA_TRY(cudaStreamSynchronize(ctx->copy_stream));
  if (ctx->oz) return lsd_ozaki_check(ctx);
  return LSD_OK;
}
int lsd_last_elapsed_ms(const lsd_ctx* ctx, double* ms) {
  if (!ctx || !ms) return LSD_EARG;
  *ms = ctx->last_ms;
  return LSD_OK;
}
int lsd_selftest(lsd_ctx* ctx, int which, double* result) {
  if (!ctx || !result) return LSD_EARG;
  CUDA_TRY(cudaSetDevice(ctx->dev));
  if (which == 0) return lsd_umma_selftest(ctx, result);
  return LSD_EARG;
}

int lsd_kernel_launches(const lsd_ctx* ctx, long long* count) {
  if (!ctx || !count) return LSD_EARG;
  *count = ctx->launches;
  return LSD_OK;
}

}  // extern "C"
