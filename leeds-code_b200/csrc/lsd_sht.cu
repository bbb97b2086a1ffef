// lsd_sht.cu -- FP64 associated-Legendre contractions on the Gauss half grid.
//
// Synthesis (spectral -> theta-Fourier) restates the _loop_sumth accumulations of
// tra_spec2phys / tra_qst2rtp / tra_grad (transform.fftw3.F90:472-520, 719-818,
// 955-1000): for each m, Y(j, m, parity) += c_lm * table(j, lm), then the north/south
// recombination Y_even +- Y_odd.  Analysis restates the parity fold and Gauss
// quadrature of tra_phys2spec / tra_leg_trans_p2s_native / tra_rtp2qst
// (transform.fftw3.F90:527-602, 825-949).
//
// Data layouts: spectral [n][H] complex (harmonic fastest, the reference's `spec`
// order); theta-Fourier rows folded into even/odd half-grid sums: synthesis writes them in
// half-row pairs for the FFT (four_off: [n][h/2][m-counter][E/O][h%2]), analysis reads them
// counter-major (four_off_a: [m-counter][n][h][E/O]);
// tables [nh][Th2] (the reference's leg_*(Th2, 0:H-1)).
//
// Synthesis CTA = (m-counter, NT shells, group); thread = one theta row j of the half
// grid, holding E/O accumulators for NT shells x 3 outputs; coefficients of the current
// k-chunk are smem broadcasts, table rows are read conflict-free along j.
// Analysis CTA = (folded column = two m-counters, NT shells, group); thread = one
// harmonic k of the column; the folded (E/O) data of a j-chunk are smem broadcasts.
#include "lsd_common.cuh"

namespace {

constexpr int S_NT = 4;   // shells per synthesis CTA
constexpr int S_KC = 16;  // harmonics per synthesis k-chunk
constexpr int A_NT = 8;   // shells per analysis CTA
constexpr int A_JC = 16;  // theta rows per analysis j-chunk
constexpr int DROW = A_JC * A_NT + 1;  // padded analysis data row (double2)

struct SynthArgs {
  int N, H, Th, Th2, NM, HB, ngroup;
  const int* mstart;
  const int* mlen;
  const int* hs;
  const double* leg;  // 8 tables [t][H][Th2]
  const double* rinv; // 1/r per shell
  SynthGroup g[6];
};

__device__ __forceinline__ double2 cmul_i(double2 a) { return make_double2(-a.y, a.x); }     // i*a
__device__ __forceinline__ double2 cmul_mi(double2 a) { return make_double2(a.y, -a.x); }    // -i*a

// KIND-specific: number of inputs, outputs and tables used
template <int KIND> struct SK;
template <> struct SK<SK_VECTOR> { static constexpr int nin = 3, nout = 3, ntab = 3; };
template <> struct SK<SK_SCALAR> { static constexpr int nin = 1, nout = 1, ntab = 1; };
template <> struct SK<SK_GRAD3> { static constexpr int nin = 2, nout = 3, ntab = 3; };
template <> struct SK<SK_GRAD2> { static constexpr int nin = 1, nout = 2, ntab = 2; };

template <int KIND>
__device__ __forceinline__ int synth_table(int t) {
  if (KIND == SK_VECTOR) return t == 0 ? LSD_LEG_P : (t == 1 ? LSD_LEG_LLP_ : LSD_LEG_LLSIN1MP);
  if (KIND == SK_SCALAR) return LSD_LEG_P;
  if (KIND == SK_GRAD3) return t == 0 ? LSD_LEG_P : (t == 1 ? LSD_LEG_P_ : LSD_LEG_SIN1MP);
  return t == 0 ? LSD_LEG_P_ : LSD_LEG_SIN1MP;  // SK_GRAD2
}

// One harmonic k of the current chunk: accumulate into the even (E) / odd (O) sums of
// the outputs; S = parity of (l + m) of this harmonic.
template <int KIND, int S, int NOUT>
__device__ __forceinline__ void synth_accum(double2 (&acc)[NOUT][2][S_NT], const double* tab,
                                            const double2* coef, int kk, int j, int Th2) {
  constexpr int O = 1 - S;
  if (KIND == SK_VECTOR) {
    const double P = tab[(0 * S_KC + kk) * Th2 + j];
    const double A1 = tab[(1 * S_KC + kk) * Th2 + j];
    const double A2 = tab[(2 * S_KC + kk) * Th2 + j];
#pragma unroll
    for (int q = 0; q < S_NT; ++q) {
      const double2 cq = coef[(0 * S_KC + kk) * S_NT + q];
      const double2 cs = coef[(1 * S_KC + kk) * S_NT + q];
      const double2 ct = coef[(2 * S_KC + kk) * S_NT + q];
      const double2 c2 = cmul_mi(ct);  // (t.Im, -t.Re)
      const double2 c3 = cmul_i(cs);   // (-s.Im, s.Re)
      // r: P on parity S ; th: llP_ on 1-S, llsin1mP on S ; ph: llsin1mP on S, llP_ on 1-S
      acc[0][S][q].x += cq.x * P;  acc[0][S][q].y += cq.y * P;
      acc[1][O][q].x += cs.x * A1; acc[1][O][q].y += cs.y * A1;
      acc[1][S][q].x += c2.x * A2; acc[1][S][q].y += c2.y * A2;
      acc[2][S][q].x += c3.x * A2; acc[2][S][q].y += c3.y * A2;
      acc[2][O][q].x += ct.x * A1; acc[2][O][q].y += ct.y * A1;
    }
  } else if (KIND == SK_SCALAR) {
    const double P = tab[kk * Th2 + j];
#pragma unroll
    for (int q = 0; q < S_NT; ++q) {
      const double2 cq = coef[kk * S_NT + q];
      acc[0][S][q].x += cq.x * P; acc[0][S][q].y += cq.y * P;
    }
  } else if (KIND == SK_GRAD3) {
    const double P = tab[(0 * S_KC + kk) * Th2 + j];
    const double D = tab[(1 * S_KC + kk) * Th2 + j];
    const double S1 = tab[(2 * S_KC + kk) * Th2 + j];
#pragma unroll
    for (int q = 0; q < S_NT; ++q) {
      const double2 cd = coef[(0 * S_KC + kk) * S_NT + q];
      const double2 cc = coef[(1 * S_KC + kk) * S_NT + q];
      const double2 ci = cmul_i(cc);
      acc[0][S][q].x += cd.x * P;  acc[0][S][q].y += cd.y * P;
      acc[1][O][q].x += cc.x * D;  acc[1][O][q].y += cc.y * D;
      acc[2 % NOUT][S][q].x += ci.x * S1; acc[2 % NOUT][S][q].y += ci.y * S1;
    }
  } else {  // SK_GRAD2
    const double D = tab[(0 * S_KC + kk) * Th2 + j];
    const double S1 = tab[(1 * S_KC + kk) * Th2 + j];
#pragma unroll
    for (int q = 0; q < S_NT; ++q) {
      const double2 cc = coef[kk * S_NT + q];
      const double2 ci = cmul_i(cc);
      acc[0][O][q].x += cc.x * D;  acc[0][O][q].y += cc.y * D;
      acc[1 % NOUT][S][q].x += ci.x * S1; acc[1 % NOUT][S][q].y += ci.y * S1;
    }
  }
}

template <int KIND>
__global__ void __launch_bounds__(256) k_synth(SynthArgs a) {
  constexpr int NIN = SK<KIND>::nin, NOUT = SK<KIND>::nout, NTAB = SK<KIND>::ntab;
  extern __shared__ double smem[];
  const int c = blockIdx.x;
  const int n0 = blockIdx.y * S_NT;
  const SynthGroup& G = a.g[blockIdx.z];
  const int Th2 = a.Th2;
  const int kbeg = a.mstart[c], klen = a.mlen[c];
  double* tab = smem;                                   // [NTAB][S_KC][Th2]
  double2* coef = (double2*)(smem + NTAB * S_KC * Th2); // [NIN][S_KC][S_NT]
  __shared__ int spar[S_KC];
  const int j = threadIdx.x;
  // accumulators acc[out][parity][shell]
  double2 acc[NOUT][2][S_NT];
#pragma unroll
  for (int o = 0; o < NOUT; ++o)
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int q = 0; q < S_NT; ++q) acc[o][p][q] = make_double2(0.0, 0.0);

  for (int k0 = 0; k0 < klen; k0 += S_KC) {
    const int kc = min(S_KC, klen - k0);
    __syncthreads();
    for (int i = threadIdx.x; i < NTAB * kc * Th2; i += blockDim.x) {
      int t = i / (kc * Th2), rem = i % (kc * Th2), kk = rem / Th2, jj = rem % Th2;
      tab[(t * S_KC + kk) * Th2 + jj] =
          a.leg[(size_t)synth_table<KIND>(t) * a.H * Th2 + (size_t)(kbeg + k0 + kk) * Th2 + jj];
    }
    for (int i = threadIdx.x; i < NIN * kc * S_NT; i += blockDim.x) {
      int f = i / (kc * S_NT), rem = i % (kc * S_NT), q = rem / kc, kk = rem % kc;
      int n = n0 + q;
      double2 v = make_double2(0.0, 0.0);
      if (n < a.N) {
        v = G.in[f][(size_t)n * a.H + kbeg + k0 + kk];
        if (KIND == SK_GRAD3 && f == 1) { double r1 = a.rinv[n]; v.x *= r1; v.y *= r1; }
        if (KIND == SK_GRAD2) { double r1 = a.rinv[n]; v.x *= r1; v.y *= r1; }
      }
      coef[(f * S_KC + kk) * S_NT + q] = v;
    }
    if (threadIdx.x < kc) spar[threadIdx.x] = a.hs[kbeg + k0 + threadIdx.x];
    __syncthreads();
    if (j < Th2) {
      for (int kk = 0; kk < kc; ++kk) {
        // parity is uniform across the block for a given k: branch so that every
        // accumulator index is a compile-time constant (registers, no local memory)
        if (spar[kk] == 0)
          synth_accum<KIND, 0>(acc, tab, coef, kk, j, Th2);
        else
          synth_accum<KIND, 1>(acc, tab, coef, kk, j, Th2);
      }
    }
  }
  if (j >= Th2) return;
#pragma unroll
  for (int o = 0; o < NOUT; ++o)
#pragma unroll
    for (int q = 0; q < S_NT; ++q) {
      int n = n0 + q;
      if (n >= a.N) continue;
      G.out[o][four_off(n, c, 0, j, a.NM, a.HB)] = acc[o][0][q];  // E
      G.out[o][four_off(n, c, 1, j, a.NM, a.HB)] = acc[o][1][q];  // O
    }
}

struct AnalArgs {
  int N, H, Th, Th2, NM, HB, Hr, ngroup;
  const int* perm;     // [Hc][Hr]: thread -> harmonic of the column, sorted by (m-counter, parity)
  const int* mstart;   // per m-counter
  const int* mlen;
  const int* hs;
  const int* hm;
  const double* leg;
  AnalGroup g[4];
};

template <int KIND>
__global__ void __launch_bounds__(288) k_anal(AnalArgs a) {
  constexpr int NF = (KIND == AK_VECTOR) ? 3 : 1;
  constexpr int NTAB = (KIND == AK_VECTOR) ? 3 : 1;
  extern __shared__ double smem[];
  const int col = blockIdx.x;        // folded column: m-counters 2col, 2col+1
  const int n0 = blockIdx.y * A_NT;
  const AnalGroup& G = a.g[blockIdx.z];
  const int Th = a.Th, Th2 = a.Th2, Hr = a.Hr;
  const int c0 = 2 * col, c1 = 2 * col + 1;
  const int len0 = a.mlen[c0];
  const int kbeg = a.mstart[c0];     // the column's harmonics are contiguous
  double* tab = smem;                                         // [NTAB][A_JC][Hr]
  double2* dat = (double2*)(smem + NTAB * A_JC * Hr);         // [2 cnt][NF][2 par][A_JC*A_NT + 1]
  // threads are ordered by (m-counter, parity) so that a warp reads one data row (a smem
  // broadcast); rows are padded by one element so that neighbouring rows use other banks
  const bool active = threadIdx.x < Hr;
  const int k = active ? a.perm[(size_t)col * Hr + threadIdx.x] : 0;
  const int cl = (k < len0) ? 0 : 1;
  const int s = active ? a.hs[kbeg + k] : 0;
  double2 acc[NF][A_NT];
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int q = 0; q < A_NT; ++q) acc[f][q] = make_double2(0.0, 0.0);
  const int tabid[3] = {LSD_LEG_GWP, LSD_LEG_GWLLP_, LSD_LEG_GWLLSIN1MP};

  for (int j0 = 0; j0 < Th2; j0 += A_JC) {
    const int jc = min(A_JC, Th2 - j0);
    __syncthreads();
    for (int i = threadIdx.x; i < NTAB * jc * Hr; i += blockDim.x) {
      int t = i / (jc * Hr), rem = i % (jc * Hr), kk = rem / jc, jj = rem % jc;
      tab[(t * A_JC + jj) * Hr + kk] = a.leg[(size_t)tabid[t] * a.H * Th2 + (size_t)(kbeg + kk) * Th2 + j0 + jj];
    }
    for (int i = threadIdx.x; i < 2 * NF * A_NT * jc; i += blockDim.x) {
      int jj = i % jc, rem = i / jc, q = rem % A_NT, rem2 = rem / A_NT, f = rem2 % NF, cc = rem2 / NF;
      int n = n0 + q;
      double2 e = make_double2(0.0, 0.0), o = e;
      if (n < a.N) {  // folded E/O data (the FFT stage folded the two hemispheres)
        const int cn = cc ? c1 : c0, j = j0 + jj;
        e = G.in[f][four_off_a(n, cn, 0, j, a.N, Th2)];
        o = G.in[f][four_off_a(n, cn, 1, j, a.N, Th2)];
      }
      dat[((cc * NF + f) * 2 + 0) * DROW + jj * A_NT + q] = e;
      dat[((cc * NF + f) * 2 + 1) * DROW + jj * A_NT + q] = o;
    }
    __syncthreads();
    if (active) {
      for (int jj = 0; jj < jc; ++jj) {
        if (KIND == AK_VECTOR) {
          const double gP = tab[(0 * A_JC + jj) * Hr + k];
          const double A1 = tab[(1 * A_JC + jj) * Hr + k];
          const double A2 = tab[(2 * A_JC + jj) * Hr + k];
          const double2* Yr_s = dat + ((cl * NF + 0) * 2 + s) * DROW + jj * A_NT;
          const double2* Yt_s = dat + ((cl * NF + 1) * 2 + s) * DROW + jj * A_NT;
          const double2* Yt_o = dat + ((cl * NF + 1) * 2 + (1 - s)) * DROW + jj * A_NT;
          const double2* Yp_s = dat + ((cl * NF + 2) * 2 + s) * DROW + jj * A_NT;
          const double2* Yp_o = dat + ((cl * NF + 2) * 2 + (1 - s)) * DROW + jj * A_NT;
#pragma unroll
          for (int q = 0; q < A_NT; ++q) {
            const double2 yr = Yr_s[q], yts = Yt_s[q], yto = Yt_o[q], yps = Yp_s[q], ypo = Yp_o[q];
            acc[0][q].x += yr.x * gP;
            acc[0][q].y += yr.y * gP;
            acc[1][q].x += yto.x * A1 + yps.y * A2;
            acc[1][q].y += yto.y * A1 - yps.x * A2;
            acc[2][q].x += ypo.x * A1 - yts.y * A2;
            acc[2][q].y += ypo.y * A1 + yts.x * A2;
          }
        } else {
          const double gP = tab[jj * Hr + k];
          const double2* Y = dat + ((cl * NF + 0) * 2 + s) * DROW + jj * A_NT;
#pragma unroll
          for (int q = 0; q < A_NT; ++q) {
            acc[0][q].x += Y[q].x * gP;
            acc[0][q].y += Y[q].y * gP;
          }
        }
      }
    }
  }
  if (!active) return;
  const int nh = kbeg + k;
  const bool m0 = a.hm[nh] == 0;
#pragma unroll
  for (int q = 0; q < A_NT; ++q) {
    int n = n0 + q;
    if (n >= a.N) continue;
    size_t id = (size_t)n * a.H + nh;
    if (KIND == AK_VECTOR) {
      G.out[0][id] = acc[0][q];  // q%Im of m = 0 is kept (transform.fftw3.F90:869)
      G.out[1][id] = make_double2(acc[1][q].x, m0 ? 0.0 : acc[1][q].y);
      G.out[2][id] = make_double2(acc[2][q].x, m0 ? 0.0 : acc[2][q].y);
    } else {
      G.out[0][id] = make_double2(acc[0][q].x, m0 ? 0.0 : acc[0][q].y);
    }
  }
}

template <int KIND>
int launch_synth_kind(lsd_ctx* ctx, const SynthGroup* groups, int ngroups) {
  SynthArgs a;
  a.N = ctx->N; a.H = ctx->H; a.Th = ctx->Th; a.Th2 = ctx->Th2; a.NM = ctx->NM; a.HB = ctx->HB;
  a.mstart = ctx->d_mstart; a.mlen = ctx->d_mlen; a.hs = ctx->d_s; a.leg = ctx->d_leg;
  a.rinv = ctx->d_rinv;
  int ng = 0;
  for (int i = 0; i < ngroups; ++i)
    if (groups[i].kind == KIND) a.g[ng++] = groups[i];
  if (ng == 0) return LSD_OK;
  a.ngroup = ng;
  constexpr int NIN = SK<KIND>::nin, NTAB = SK<KIND>::ntab;
  size_t smem = sizeof(double) * NTAB * S_KC * ctx->Th2 + sizeof(double2) * NIN * S_KC * S_NT;
  cudaFuncSetAttribute(k_synth<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_synth<KIND>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  int threads = ((ctx->Th2 + 31) / 32) * 32;
  dim3 grid(ctx->NM, ceil_div(ctx->N, S_NT), ng);
  k_synth<KIND><<<grid, threads, smem, ctx->stream>>>(a);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_synth: ") + cudaGetErrorString(e));
  return LSD_OK;
}

template <int KIND>
int launch_anal_kind(lsd_ctx* ctx, const AnalGroup* groups, int ngroups) {
  AnalArgs a;
  a.N = ctx->N; a.H = ctx->H; a.Th = ctx->Th; a.Th2 = ctx->Th2; a.NM = ctx->NM; a.HB = ctx->HB; a.Hr = ctx->Hr;
  a.mstart = ctx->d_mstart; a.mlen = ctx->d_mlen; a.hs = ctx->d_s; a.hm = ctx->d_m; a.leg = ctx->d_leg;
  int ng = 0;
  for (int i = 0; i < ngroups; ++i)
    if (groups[i].kind == KIND) a.g[ng++] = groups[i];
  if (ng == 0) return LSD_OK;
  a.ngroup = ng;
  constexpr int NF = (KIND == AK_VECTOR) ? 3 : 1;
  size_t smem = sizeof(double) * NF * A_JC * ctx->Hr + sizeof(double2) * 2 * NF * 2 * DROW;
  a.perm = ctx->d_aperm;
  cudaFuncSetAttribute(k_anal<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_anal<KIND>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  int threads = ((ctx->Hr + 31) / 32) * 32;
  if (threads > 1024) return lsd_fail(ctx, LSD_EARG, "analysis: folded column longer than 1024 harmonics");
  dim3 grid(ctx->Hc, ceil_div(ctx->N, A_NT), ng);
  k_anal<KIND><<<grid, threads, smem, ctx->stream>>>(a);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lsd_fail(ctx, LSD_ECUDA, std::string("k_anal: ") + cudaGetErrorString(e));
  return LSD_OK;
}

}  // namespace

int lsd_launch_synth(lsd_ctx* ctx, const SynthGroup* groups, int ngroups) {
  if (ctx->oz) return lsd_ozaki_launch_synth(ctx, groups, ngroups);  // LSD_PREC_OZAKI
  int rc;
  if ((rc = launch_synth_kind<SK_VECTOR>(ctx, groups, ngroups))) return rc;
  if ((rc = launch_synth_kind<SK_SCALAR>(ctx, groups, ngroups))) return rc;
  if ((rc = launch_synth_kind<SK_GRAD3>(ctx, groups, ngroups))) return rc;
  if ((rc = launch_synth_kind<SK_GRAD2>(ctx, groups, ngroups))) return rc;
  return LSD_OK;
}

int lsd_launch_anal(lsd_ctx* ctx, const AnalGroup* groups, int ngroups) {
  if (ctx->oz) return lsd_ozaki_launch_anal(ctx, groups, ngroups);  // LSD_PREC_OZAKI
  int rc;
  if ((rc = launch_anal_kind<AK_VECTOR>(ctx, groups, ngroups))) return rc;
  if ((rc = launch_anal_kind<AK_SCALAR>(ctx, groups, ngroups))) return rc;
  return LSD_OK;
}
