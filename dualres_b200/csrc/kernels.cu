// Device kernels of the dual-resolution GP-HMC sampler.
//
// The sampler keeps every chain's state in the spectral domain of the
// circulant embedding: u = IFFT(mu) and q = IFFT(p) (unnormalised).  In that
// basis the reference's operators (include/dualres/MultiResParameters.h) become:
//   position update  mu* += FFT(IFFT(p) eps/(N lambda_m))  ->  u* += eps q / lambda_m
//   prior gradient   FFT(IFFT(mu)/(-N lambda))             ->  -u / lambda
//   log prior        -(1/2N) sum |IFFT(mu)|^2 / lambda       ->  -(1/2N) sum |u|^2 / lambda
//   kinetic energy   -(1/2N) sum |IFFT(p)|^2 / lambda_m      ->  -(1/2N) sum |q|^2 / lambda_m
// all element-wise, zeroed on S = {Re lambda <= 0} exactly as _low_rank_adjust
// does.  Only the data term needs real space: Re mu at the data voxels, and the
// scatter of the data gradient.  One gradient therefore costs one pruned
// forward transform (spectral -> real box) and one pruned inverse transform
// (real box -> spectral) instead of the reference's four full 3D FFTs.
#include "common.cuh"
#include "drb.h"
#include "fft.cuh"
#include "tma.cuh"

namespace drb {

// e / d as __umulhi(e, box_div_magic(d)) for box positions (e < 2^15, 2 <= d <= 1024): the multiplier
// ceil(2^32 / d) gives the exact quotient there, without a division per element.
__device__ __forceinline__ uint32_t box_div_magic(int d) { return 0xFFFFFFFFu / (uint32_t)d + 1u; }

// ----------------------------------------------------------------- twiddles
__device__ float2 g_tw_f[TW_TOTAL];
__device__ double2 g_tw_d[TW_TOTAL];

// ----------------------------------------------------------------- HMC parameters
// Device restatement of HMCParameters<float> (include/dualres/HMCParameters.h).
__device__ __forceinline__ float hmc_eps(const ChainState& h, double u01) {
  // :212-221  eps() = eps (warm-up) or max(eps * U(0.9, 1.1), eps0)
  if (h.warmup) return (float)h.eps;
  return (float)fmax(h.eps * (0.9 + 0.2 * u01), h.eps0);
}
__device__ __forceinline__ int hmc_steps(const ChainState& h) {  // :172-179
  return h.eps_start_found ? h.integrator_steps : 1;
}
__device__ __forceinline__ int hmc_save_iteration(const ChainState& h) {  // :158-161
  return (h.iteration > h.burnin) && ((h.iteration - h.burnin) % h.thin == 0);
}
__device__ void hmc_update(ChainState& h, float mh_rate_f) {  // :259-297
  const double mh_rate = (double)mh_rate_f;
  if (h.iteration == h.burnin) {
    h.warmup = 0;
    h.eps_start_found = 1;
    if (h.eps_bar > h.eps0) h.eps = h.eps_bar;
  }
  if (h.warmup) {
    if (!h.eps_start_found) {
      if (h.iteration == 0) h.A = 2 * (int)(mh_rate > 0.5) - 1;
      if (pow(mh_rate, h.A) > pow(2.0, -h.A)) {
        h.eps *= pow(2.0, h.A);
      } else {
        h.eps_start_found = 1;
        h.eps_target = log(10.0 * h.eps);
      }
    } else {
      const double it = (double)h.iteration;
      h.h_bar = (1 - 1 / (it + h.t0)) * h.h_bar + (h.mh_target - mh_rate) / (it + h.t0);
      h.eps = exp(h.eps_target - (double)sqrtf((float)h.iteration) * h.h_bar / h.gamma);
      h.eps = fmax(h.eps, h.eps0);
      const double pk = pow((double)(float)h.iteration, -h.kappa);
      h.eps_bar = exp(pk * log(h.eps) + (1 - pk) * log(h.eps_bar));
    }
  } else {
    h.mh_running_sum += mh_rate;
  }
  h.iteration++;
}

// Marsaglia & Tsang (2000), "A simple method for generating gamma variables",
// ACM TOMS 26(3); shape < 1 by Gamma(a) = Gamma(a + 1) U^(1/a).  Draws come
// from the counter stream (stream, chain, iteration, base + attempt).  The
// loop is bounded; a failure sets *err and returns the mean.
__device__ double gamma_draw(double shape, double scale, uint64_t seed, uint32_t stream, uint32_t chain,
                             uint32_t iter, uint32_t base, int* err) {
  double boost = 1.0;
  if (shape < 1.0) {
    const u32x4 r = philox(u32x4{base + 1000u, iter, chain, stream}, seed);
    boost = pow(u01d(r.x, r.y), 1.0 / shape);
    shape += 1.0;
  }
  const double d = shape - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
  for (uint32_t a = 0; a < 64; a++) {
    const u32x4 r1 = philox(u32x4{base + 2 * a, iter, chain, stream}, seed);
    const u32x4 r2 = philox(u32x4{base + 2 * a + 1, iter, chain, stream}, seed);
    const double x = box_muller_d(u01d(r1.x, r1.y), u01d(r1.z, r1.w)).x;
    double v = 1.0 + c * x;
    if (v <= 0.0) continue;
    v = v * v * v;
    const double u = u01d(r2.x, r2.y);
    if (log(u) < 0.5 * x * x + d - d * v + d * log(v)) return d * v * boost * scale;
  }
  *err += 1;
  return shape * scale;
}

// ----------------------------------------------------------------- pass kernel
// Batched 1D FFT along the middle axis of [A][n][B] arrays, one tile of 32
// lines (line = a * B + b) per block.  CPB = 1: the 32 lines of one chain
// (blockIdx.y).  CPB = 8: 4 consecutive lines of 8 chains (chain group
// blockIdx.y), used by the z passes whose epilogue / prologue touch the
// chain-minor arrays mu_D, mu_O and gD: a warp then reads and writes 8 chains
// x 4 bytes contiguously there, instead of one 4-byte value per 256-byte row,
// while its T2 accesses stay whole 32-byte sectors (4 lines x 8 bytes).
template <int N> struct PassCfg {
  static constexpr int NT = N >= 512 ? 512 : 256;
};

template <int N, int DIR, int PRO, int EPI, class C, int CPB = 1, int PLAN = 0>
__global__ void __launch_bounds__(PassCfg<N>::NT) k_pass(PassArgs a, DevVolume v, DevChains ch, const C* __restrict__ tw) {
  grid_dep_wait();
  constexpr int TL = TILE_LINES, P = TILE_LINES + 1, NT = PassCfg<N>::NT, LPC = TILE_LINES / CPB;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  __shared__ int s_ok[CPB], s_hsel[CPB], s_wo[CPB];
  __shared__ long long s_in0[TL], s_out0[TL];  // per tile line: index of its element 0 in the input / output
  const int cbase = CPB == 1 ? ((a.chain_only >= 0) ? a.chain_only : (int)blockIdx.y) : (int)blockIdx.y * CPB;
  if (threadIdx.x < CPB) {
    // per chain of the tile: active at this step, the half of mu_D / mu_O written, whether mu_O is written
    const int c = cbase + (int)threadIdx.x;
    int ok = CPB == 1 || c < ch.C;
    if (ok && a.step >= 0 && ch.st != nullptr && a.step > ch.st[c].L_cur) ok = 0;
    s_ok[threadIdx.x] = ok;
    int hs = 0, wo = 0;
    if (EPI == EPI_GATHER && ok) {
      hs = (ch.st != nullptr ? ch.st[c].acc : 0) ^ a.sel;
      wo = a.write_o == 1 || (a.write_o == 2 && ch.st != nullptr && a.step == ch.st[c].L_cur);
    }
    s_hsel[threadIdx.x] = hs;
    s_wo[threadIdx.x] = wo;
  }
  const long long lines = (long long)a.A * a.B;
  const long long l0 = (long long)blockIdx.x * LPC;
  const int B = a.B, n_in = a.n_in, n_out = a.n_out;
  if (threadIdx.x < TL) {
    // line lam = a * B + b starts at (a * n) * B + b; computed once per line rather than per element
    const long long lam = l0 + threadIdx.x % LPC;
    const long long aa = lam / B, bb = lam - aa * B;
    s_in0[threadIdx.x] = aa * n_in * B + bb;
    s_out0[threadIdx.x] = aa * n_out * B + bb;
  }
  __syncthreads();
  if (CPB == 1 && !s_ok[0]) return;
  const int nl = (int)min((long long)LPC, lines - l0);
  // tile line l: chain slot l / LPC of the tile, line l0 + l % LPC
  auto valid = [&](int l) { return (l % LPC) < nl && s_ok[l / LPC]; };
  auto chain = [&](int l) { return cbase + l / LPC; };
  auto in_index = [&](int l, int i) -> long long { return s_in0[l] + (long long)i * B; };
  auto out_index = [&](int l, int k) -> long long { return s_out0[l] + (long long)k * B; };
  // bounds of the data-dependent indices (checked builds only): a chain's stride in the input / output (the whole
  // array when there is one field), the box, the data and output voxels
  const long long in_lim = a.in_cs > 0 ? a.in_cs : 0x7fffffffffffffffLL;
  const long long out_lim = a.out_cs > 0 ? a.out_cs : 0x7fffffffffffffffLL;
  const long long box = (long long)v.bx * v.by * v.bz;
  auto load = [&](int l, int i) -> C {
    C val = mk((decltype(C().x))0, (decltype(C().x))0);
    if (valid(l) && i < n_in) {
      const long long idx = in_index(l, i);
      const int c = chain(l);
      if (PRO == PRO_LOAD) {
        // the forward z pass is the last reader of its input (T2): streaming loads, evicted first
        if (in_bounds(idx, in_lim, ch.err)) {
          if constexpr (EPI == EPI_GATHER) val = __ldcs(reinterpret_cast<const C*>(a.in) + (long long)c * a.in_cs + idx);
          else val = reinterpret_cast<const C*>(a.in)[(long long)c * a.in_cs + idx];
        }
      } else if (in_bounds(idx, box, ch.err)) {
        const int j = v.box_to_d[idx];
        if (j >= 0 && in_bounds(j, v.n_h, ch.err)) val.x = ch.gD[(long long)j * ch.Cp + c];
      }
    }
    return val;
  };
  // the loads of a thread are issued before its shared-memory stores, up to 16 at a time: PER independent loads in
  // flight per round (tiles of a whole number of block-widths)
  constexpr int PER = TL * N / NT;
  constexpr int CH = PER > 16 ? 16 : PER;
  if constexpr (PER >= 1 && PER * NT == TL * N && PER % CH == 0) {
#pragma unroll 1
    for (int k0 = 0; k0 < PER; k0 += CH) {
      C r[CH];
#pragma unroll
      for (int k = 0; k < CH; k++) {
        const int e = threadIdx.x + (k0 + k) * NT;
        r[k] = B == 1 ? load(e / N, e % N) : load(e % TL, e / TL);
      }
#pragma unroll
      for (int k = 0; k < CH; k++) {
        const int e = threadIdx.x + (k0 + k) * NT;
        if (B == 1) sm[(e % N) * P + e / N] = r[k];
        else sm[(e / TL) * P + e % TL] = r[k];
      }
    }
  } else if (B == 1) {
    for (int e = threadIdx.x; e < TL * N; e += NT) {
      const int l = e / N, i = e % N;
      sm[i * P + l] = load(l, i);
    }
  } else {
    for (int e = threadIdx.x; e < TL * N; e += NT) {
      const int i = e / TL, l = e % TL;
      sm[i * P + l] = load(l, i);
    }
  }
  __syncthreads();
  fft_smem<N, DIR, TL, NT, C, PLAN>(sm, 1, P, TL, tw + tw_offset(N));

  const auto scale = (decltype(C().x))a.scale;
  auto store = [&](int l, int k) {
    if (!valid(l) || k >= n_out) return;
    const long long idx = out_index(l, k);
    const int c = chain(l);
    const C val = sm[k * P + l];
    if (EPI == EPI_STORE) {
      if (in_bounds(idx, out_lim, ch.err))
        reinterpret_cast<C*>(a.out)[(long long)c * a.out_cs + idx] = mk(val.x * scale, val.y * scale);
    } else if (in_bounds(idx, box, ch.err)) {
      const int slot = l / LPC;
      const int j = v.box_to_d[idx];
      if (j >= 0 && in_bounds(j, v.n_h, ch.err))
        ch.muD[((long long)s_hsel[slot] * v.n_h + j) * ch.Cp + c] = (float)(val.x * scale);
      if (s_wo[slot]) {
        const int o = v.box_to_o[idx];
        if (o >= 0 && in_bounds(o, v.n_o, ch.err))
          ch.muO[((long long)s_hsel[slot] * v.n_o + o) * ch.Cp + c] = (float)(val.x * scale);
      }
    }
  };
  if (B == 1) {
    for (int e = threadIdx.x; e < TL * N; e += NT) store(e / N, e % N);
  } else {
    for (int e = threadIdx.x; e < TL * N; e += NT) store(e % TL, e / TL);
  }
}

// ----------------------------------------------------------------- x-line kernel
// The hot kernel of one leapfrog step, for 32 x-lines of one chain:
//   inverse x-FFT of the data gradient (spectral except along x),
//   kick  q += k eps (IFFT(data grad) - u / lambda)          (MultiResParameters.h:690, 699)
//   drift u* += eps q / lambda_m                              (:693-698)
//   forward x-FFT of u* for the next gradient.
// Step 0 also draws the momentum (:784-815) and the initial energies; the
// last step only kicks and accumulates the final energies (:702-705).
template <int E0> struct XCfg {
  static constexpr int NT = E0 >= 512 ? 512 : 256;
  // blocks per SM the register budget targets: at E0 = 256 the 67.6 KB tile allows three (85 registers, no
  // spills; two at the unconstrained 126 registers), at E0 <= 128 four
  static constexpr int MINB = E0 >= 512 ? 1 : (E0 == 256 ? 3 : 4);
};

template <int E0, int PLAN = 0>
__global__ void __launch_bounds__(XCfg<E0>::NT, XCfg<E0>::MINB) k_xline(DevVolume v, DevChains ch, int step, int flags,
                                                        const float2* __restrict__ tw) {
  grid_dep_wait();
  constexpr int TL = TILE_LINES, P = TILE_LINES + 1, NT = XCfg<E0>::NT;
  extern __shared__ __align__(16) unsigned char smraw[];
  float2* sm = reinterpret_cast<float2*>(smraw);
  __shared__ double red[NT / 32];
  const int c = blockIdx.y;
  const ChainState& st = ch.st[c];
  const int Lc = st.L_cur;
  if (step > Lc) return;
  const bool first = step == 0, last = step == Lc;
  const float eps = st.eps_cur, sh = st.sh;
  const int acc = st.acc;
  const long long N = v.N;
  const long long lines = (long long)v.E1 * v.E2;
  const long long lam0 = (long long)blockIdx.x * TL;
  // the block's lines of the state and of T1 lie in their arrays (checked builds)
  if (!in_bounds(min(lam0 + TL, lines) * E0 - 1, N, ch.err) ||
      !in_bounds(min(lam0 + TL, lines) * v.bx - 1, ch.t1_stride, ch.err))
    return;
  const int nl = (int)min((long long)TL, lines - lam0);
  float2* Ub = ch.U + (long long)c * 2 * N;
  const float2* Usrc = Ub + (long long)(first ? acc : (acc ^ 1)) * N;
  float2* Udst = Ub + (long long)(acc ^ 1) * N;
  float2* Qc = ch.Q + (long long)c * N;
  float2* T1 = ch.T1 + (long long)c * ch.t1_stride;
  const int bx = v.bx;
  if ((flags & XF_L2_PREFETCH) && threadIdx.x == 0 && E0 >= 4) {
    const bool draw = first && !(flags & XF_FIXED_MOMENTUM);
    bulk_prefetch_l2(Usrc + lam0 * E0, (uint32_t)nl * E0 * 8);
    if (!draw) bulk_prefetch_l2(Qc + lam0 * E0, (uint32_t)nl * E0 * 8);
    bulk_prefetch_l2(v.sinv + lam0 * E0, (uint32_t)nl * E0 * 4);
  }

  for (int e = threadIdx.x; e < TL * E0; e += NT) {
    const int l = e / E0, x = e % E0;
    float2 val = make_float2(0.f, 0.f);
    if (l < nl && x < bx) val = T1[(lam0 + l) * bx + x];
    sm[x * P + l] = val;
  }
  __syncthreads();
  fft_smem<E0, +1, TL, NT, float2, PLAN>(sm, 1, P, TL, tw + tw_offset(E0));

  const bool fixed = (flags & XF_FIXED_MOMENTUM) != 0;
  const bool write_q = !last || (flags & XF_WRITE_Q_LAST);
  const float keps = ((first || last) ? 0.5f : 1.0f) * eps;
  const float Nf = (float)N;
  double pa = 0.0, pb = 0.0;
  for (int e = threadIdx.x; e < TL * (E0 / 2); e += NT) {
    const int l = e / (E0 / 2), x = 2 * (e % (E0 / 2));
    if (l >= nl) continue;
    const long long gi = (lam0 + l) * E0 + x;
    const float4 u4 = __ldcs(reinterpret_cast<const float4*>(Usrc + gi));
    const float2 s2 = *reinterpret_cast<const float2*>(v.sinv + gi);
    float4 q4;
    float2 w0 = make_float2(0.f, 0.f), w1 = w0;
    if (first && !fixed) {
      const u32x4 r = philox(u32x4{(uint32_t)(gi >> 1), (uint32_t)st.iteration, (uint32_t)(ch.chain0 + c),
                                   RNG_MOMENTUM}, ch.seed);
      w0 = box_muller(u01f(r.x), u01f(r.y));
      w1 = box_muller(u01f(r.z), u01f(r.w));
      pa += (double)(w0.x * w0.x + w0.y * w0.y) + (double)(w1.x * w1.x + w1.y * w1.y);
    } else {
      q4 = __ldcs(reinterpret_cast<const float4*>(Qc + gi));
    }
    float2 uo[2], qo[2];
#pragma unroll
    for (int m = 0; m < 2; m++) {
      const float2 u = m == 0 ? make_float2(u4.x, u4.y) : make_float2(u4.z, u4.w);
      const float s = m == 0 ? s2.x : s2.y;
      const bool live = s > 0.0f;
      const float lm = s + sh;  // lambda_m = 1/lambda + sigma_h^-2 (MultiResParameters.h:735-738)
      float2 q;
      if (first && !fixed) {
        const float2 w = m == 0 ? w0 : w1;
        const float a = live ? sqrtf(Nf * lm) : 0.0f;
        q = make_float2(a * w.x, a * w.y);
      } else {
        q = m == 0 ? make_float2(q4.x, q4.y) : make_float2(q4.z, q4.w);
        if (first && live) pa += (double)(q.x * q.x + q.y * q.y) / (double)lm;
      }
      if (first && live) pb += (double)(u.x * u.x + u.y * u.y) * (double)s;
      const float2 g = sm[(x + m) * P + l];
      float2 gt = g;
      if (live) {
        gt.x = fmaf(-u.x, s, g.x);
        gt.y = fmaf(-u.y, s, g.y);
      }
      q.x = fmaf(keps, gt.x, q.x);
      q.y = fmaf(keps, gt.y, q.y);
      float2 un = u;
      if (last) {
        // the final energies; a step that is both first and last only evaluates (a gradient / log posterior
        // call) and keeps the energies at mu
        if (live && !first) {
          pa += (double)(u.x * u.x + u.y * u.y) * (double)s;
          pb += (double)(q.x * q.x + q.y * q.y) / (double)lm;
        }
      } else if (live) {
        const float f = eps / lm;
        un.x = fmaf(f, q.x, u.x);
        un.y = fmaf(f, q.y, u.y);
      }
      uo[m] = un;
      qo[m] = q;
      sm[(x + m) * P + l] = un;
    }
    // streaming loads and stores of the state, as in the plane kernel: it is not read again before the next step
    if (write_q) __stcs(reinterpret_cast<float4*>(Qc + gi), make_float4(qo[0].x, qo[0].y, qo[1].x, qo[1].y));
    if (!last) __stcs(reinterpret_cast<float4*>(Udst + gi), make_float4(uo[0].x, uo[0].y, uo[1].x, uo[1].y));
  }
  // per-block partial sums -> accept step
  if (first || last) {
    const double ta = block_sum(pa, red);
    if (threadIdx.x == 0) ch.part[((long long)c * NSLOT + (first ? SL_E0 : SL_LPL)) * ch.maxblk + blockIdx.x] = ta;
    const double tb = block_sum(pb, red);
    if (threadIdx.x == 0) ch.part[((long long)c * NSLOT + (first ? SL_LP0 : SL_KL)) * ch.maxblk + blockIdx.x] = tb;
  }
  if (last) return;
  __syncthreads();
  fft_smem<E0, -1, TL, NT, float2, PLAN>(sm, 1, P, TL, tw + tw_offset(E0));
  const uint32_t mb = box_div_magic(bx);
  for (int e = threadIdx.x; e < TL * bx; e += NT) {
    const int l = (int)__umulhi((uint32_t)e, mb), x = e - l * bx;
    if (l < nl) T1[(lam0 + l) * bx + x] = sm[x * P + l];
  }
}

// ----------------------------------------------------------------- xy-plane kernel
// The leapfrog update fused with the y and x transforms of one z-plane of one
// chain (E0 == E1 == E), one block per (z-plane, chain):
//   T2[c][z][y < by][x < bx] --inverse y (columns x < bx), inverse x (rows)-->
//   spectral plane; kick / drift as in k_xline; forward x, forward y --> T2.
// For E = 64 and 128 the plane uses the padded layout of PaddedPlane (bank-
// conflict free radix stages); other sizes use an odd row pitch.  With
// PREFETCH the plane's U and q planes are brought into shared memory at
// entry by bulk asynchronous copies (1D TMA, completion on an mbarrier) so
// that their DRAM latency overlaps the inverse transforms; 1/lambda, one array
// shared by every chain, stays in L2.  The wait is bounded and a time-out is
// recorded in ch.err.
template <int E>
struct PlaneGeom {
  static constexpr bool PADDED = (E == 64 || E == 128);
  static constexpr int R1 = E == 128 ? 16 : 8, R2 = 8;
  static constexpr int P = E + 1;  // odd pitch of the unpadded layout
  static constexpr int SIZE = PADDED ? PaddedPlane<E>::SIZE : E * (E + 1);
  __device__ __forceinline__ static int at(int y, int x) {
    if constexpr (PADDED) return PaddedPlane<E>::phys(y, x);
    else return y * P + x;
  }
};

// PREFETCH: the U and q planes are bulk-copied into shared memory at entry; 256 threads and 128 registers, two
// blocks per SM (E <= 64).  Without it a register budget for three blocks of 256 threads (E <= 64): 80 registers
// and 80 B of spill against 64 registers and 200 B for four, which with the state prefetched into L2 is the faster
// (64^2 plane x 64 chains 150.0 against 150.9 us, one chain 10.8 against 12.4 us).
template <int E, bool PREFETCH> struct PlaneCfg {
  static constexpr int NT = E >= 128 ? 512 : 256;
  static constexpr int MINB = PREFETCH ? 2 : (E <= 64 ? 3 : 1);  // blocks per SM the register budget targets
};

// Shared-memory layout in bytes: [mbarrier | plane | U | q].
struct PlaneLayout {
  int plane_off, u_off, q_off, total;
};
__host__ __device__ inline PlaneLayout plane_layout(int E, int plane_elems, bool prefetch) {
  PlaneLayout L;
  L.plane_off = prefetch ? 128 : 0;
  const int pe = (L.plane_off + plane_elems * 8 + 127) / 128 * 128;
  L.u_off = pe;
  L.q_off = pe + E * E * 8;
  L.total = prefetch ? L.q_off + E * E * 8 : L.plane_off + plane_elems * 8;
  return L;
}

// The padded planes prune both transforms to the box (ncols x nrows of T2): the inverse transforms read only the
// box (everything else is zero and is never stored), and the forward transforms write only what lands in it.
template <int E>
__device__ __forceinline__ void plane_fft(float2* sm, int ncols, int nrows, int dir, const float2* tw) {
  using G = PlaneGeom<E>;
  if constexpr (G::PADDED) {
    if (dir > 0) {
      plane_cols<E, G::R1, G::R2, +1>(sm, ncols, tw, nrows, E);
      plane_rows<E, G::R1, G::R2, +1>(sm, tw, ncols, E);
    } else {
      plane_rows<E, G::R1, G::R2, -1>(sm, tw, E, ncols);
      plane_cols<E, G::R1, G::R2, -1>(sm, ncols, tw, E, nrows);
    }
  } else {
    if (dir > 0) {
      fft_smem_warp<E, +1>(sm, 1, G::P, ncols, tw);
      fft_smem_warp<E, +1>(sm, G::P, 1, E, tw);
    } else {
      fft_smem_warp<E, -1>(sm, G::P, 1, E, tw);
      fft_smem_warp<E, -1>(sm, 1, G::P, ncols, tw);
    }
  }
}

// One plane of one chain after its inverse transforms, in two parts.  plane_update: the kick (and at step 0 the
// momentum draw) and the drift, with the state read from srcU / srcQ / srcS (global memory, or shared-memory copies
// of this plane) and written to Udst / Qc in global memory; the energies' per-thread partials go to pa / pb.
// need_q: the momentum is read (false only for the momentum draw at step 0).  GSRC: srcU / srcQ are in global
// memory, read with streaming loads (ld.global.cs), as the U and q stores are made; a plane's state is not read
// again before the next leapfrog step, by which time it has left L2 anyway, and evicting it first keeps T2 and the
// smaller arrays of the following kernels in L2 (5.97 against 6.04 ms per 64-chain iteration).  The shared-memory
// copies of the prefetching variant take plain loads: a global-space load of a shared address is an error.
// plane_finish: the energies' block partials, then the forward transforms and the T2 store.
template <int E, int NT, bool GSRC>
__device__ __forceinline__ void plane_update(float2* sm, const DevVolume& v, const DevChains& ch,
                                             const ChainState& st, int c, int z, bool first, bool last, bool need_q,
                                             int flags, const float2* srcU, const float2* srcQ, const float* srcS,
                                             float2* Udst, float2* Qc, double& pa_out, double& pb_out) {
  using G = PlaneGeom<E>;
  const int tid = threadIdx.x;
  const float eps = st.eps_cur, sh = st.sh;
  const bool write_q = !last || (flags & XF_WRITE_Q_LAST);
  const float keps = ((first || last) ? 0.5f : 1.0f) * eps;
  const float Nf = (float)v.N;
  double pa = 0.0, pb = 0.0;
  // Pairs of x-adjacent points: element pair e sits at li = 2e of the plane (x = 2 (e mod E/2), y = e / (E/2)),
  // so U, q and 1/lambda are read as float4 / float4 / float2 at index e.  Each thread issues the loads of B pairs
  // before computing them; with the block's state prefetched into L2 at entry one pair suffices (two pairs were
  // 154.7 against 151.8 us for a 64^2 plane x 64 chains).  A thread reads and writes only its own elements, which is
  // why the in-place state buffers may be marked non-aliasing.
  constexpr int TOTAL = E * (E / 2);
  constexpr int B = 1;
  const float4* __restrict__ gU = reinterpret_cast<const float4*>(srcU);
  const float4* __restrict__ gQ = reinterpret_cast<const float4*>(srcQ);
  const float2* __restrict__ gS = reinterpret_cast<const float2*>(srcS);
  float4* __restrict__ oQ = reinterpret_cast<float4*>(Qc);
  float4* __restrict__ oU = reinterpret_cast<float4*>(Udst);
  for (int e0 = tid; e0 < TOTAL; e0 += B * NT) {
    float4 u4v[B], q4v[B];
    float2 s2v[B];
#pragma unroll
    for (int b = 0; b < B; b++) {
      const int e = e0 + b * NT;
      if (e < TOTAL) {
        if constexpr (GSRC) {
          u4v[b] = __ldcs(gU + e);
          q4v[b] = need_q ? __ldcs(gQ + e) : make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
          u4v[b] = gU[e];
          q4v[b] = need_q ? gQ[e] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        s2v[b] = gS[e];
      }
    }
#pragma unroll
    for (int b = 0; b < B; b++) {
      const int e = e0 + b * NT;
      if (e >= TOTAL) continue;
      const int y = e / (E / 2), x = 2 * (e % (E / 2));
      const float4 u4 = u4v[b];
      const float2 s2 = s2v[b];
      const float4 q4 = q4v[b];
      float2 w0 = make_float2(0.f, 0.f), w1 = w0;
      if (!need_q) {
        const long long gi = (long long)z * E * E + 2 * e;
        const u32x4 r = philox(u32x4{(uint32_t)(gi >> 1), (uint32_t)st.iteration, (uint32_t)(ch.chain0 + c),
                                     RNG_MOMENTUM}, ch.seed);
        w0 = box_muller(u01f(r.x), u01f(r.y));
        w1 = box_muller(u01f(r.z), u01f(r.w));
        pa += (double)(w0.x * w0.x + w0.y * w0.y) + (double)(w1.x * w1.x + w1.y * w1.y);
      }
      const int pi0 = G::at(y, x), pi1 = pi0 + 1;  // x is even: x + 1 is the next slot in either layout
      float2 uo[2], qo[2];
#pragma unroll
      for (int m = 0; m < 2; m++) {
        const float2 u = m == 0 ? make_float2(u4.x, u4.y) : make_float2(u4.z, u4.w);
        const float s = m == 0 ? s2.x : s2.y;
        const bool live = s > 0.0f;
        const float lm = s + sh;
        float2 q;
        if (!need_q) {
          const float2 w = m == 0 ? w0 : w1;
          const float a = live ? sqrtf(Nf * lm) : 0.0f;
          q = make_float2(a * w.x, a * w.y);
        } else {
          q = m == 0 ? make_float2(q4.x, q4.y) : make_float2(q4.z, q4.w);
          if (first && live) pa += (double)(q.x * q.x + q.y * q.y) / (double)lm;
        }
        if (first && live) pb += (double)(u.x * u.x + u.y * u.y) * (double)s;
        const int pi = m == 0 ? pi0 : pi1;
        const float2 g = sm[pi];
        float2 gt = g;
        if (live) {
          gt.x = fmaf(-u.x, s, g.x);
          gt.y = fmaf(-u.y, s, g.y);
        }
        q.x = fmaf(keps, gt.x, q.x);
        q.y = fmaf(keps, gt.y, q.y);
        float2 un = u;
        if (last) {
          if (live && !first) {  // first and last: an evaluation step, energies at mu only
            pa += (double)(u.x * u.x + u.y * u.y) * (double)s;
            pb += (double)(q.x * q.x + q.y * q.y) / (double)lm;
          }
        } else if (live) {
          const float f = eps / lm;
          un.x = fmaf(f, q.x, u.x);
          un.y = fmaf(f, q.y, u.y);
        }
        uo[m] = un;
        qo[m] = q;
        sm[pi] = un;
      }
      if (write_q) __stcs(oQ + e, make_float4(qo[0].x, qo[0].y, qo[1].x, qo[1].y));
      if (!last) __stcs(oU + e, make_float4(uo[0].x, uo[0].y, uo[1].x, uo[1].y));
    }
  }
  pa_out = pa;
  pb_out = pb;
}

template <int E, int NT>
__device__ __forceinline__ void plane_finish(float2* sm, const DevChains& ch, int c, int z, bool first, bool last,
                                             double pa, double pb, float2* T, int bx, int by, const float2* twE,
                                             double* red) {
  using G = PlaneGeom<E>;
  const int tid = threadIdx.x;
  if (first || last) {
    const double ta = block_sum(pa, red);
    if (tid == 0) ch.part[((long long)c * NSLOT + (first ? SL_E0 : SL_LPL)) * ch.maxblk + z] = ta;
    const double tb = block_sum(pb, red);
    if (tid == 0) ch.part[((long long)c * NSLOT + (first ? SL_LP0 : SL_KL)) * ch.maxblk + z] = tb;
  }
  if (last) return;
  __syncthreads();
  plane_fft<E>(sm, bx, by, -1, twE);
  const uint32_t mb = box_div_magic(bx);
  for (int e = tid; e < by * bx; e += NT) {
    const int y = (int)__umulhi((uint32_t)e, mb), x = e - y * bx;
    T[y * bx + x] = sm[G::at(y, x)];
  }
}

// Loads the T2 box of one plane into the plane buffer (for the padded layout only the box: the pruned inverse
// transforms read nothing outside it).
template <int E, int NT>
__device__ __forceinline__ void plane_load_box(float2* sm, const float2* __restrict__ T, int bx, int by) {
  using G = PlaneGeom<E>;
  const int tid = threadIdx.x;
  if constexpr (G::PADDED) {
    const uint32_t mb = box_div_magic(bx);
    for (int e = tid; e < by * bx; e += NT) {
      const int y = (int)__umulhi((uint32_t)e, mb), x = e - y * bx;
      sm[G::at(y, x)] = __ldcs(T + e);  // the last read of this T2 plane before the next inverse z pass
    }
  } else {
    for (int e = tid; e < E * E; e += NT) {
      const int y = e / E, x = e % E;
      sm[G::at(y, x)] = (y < by && x < bx) ? T[y * bx + x] : make_float2(0.f, 0.f);
    }
  }
}

template <int E, bool PREFETCH>
__global__ void __launch_bounds__(PlaneCfg<E, PREFETCH>::NT, PlaneCfg<E, PREFETCH>::MINB) k_xyplane(DevVolume v, DevChains ch, int step, int flags,
                                                                       const float2* __restrict__ tw) {
  grid_dep_wait();
  constexpr int NT = PlaneCfg<E, PREFETCH>::NT;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ double red[NT / 32];
  const PlaneLayout Ly = plane_layout(E, PlaneGeom<E>::SIZE, PREFETCH);
  float2* sm = reinterpret_cast<float2*>(smraw + Ly.plane_off);
  const int c = blockIdx.y, z = blockIdx.x;
  const ChainState& st = ch.st[c];
  const int Lc = st.L_cur;
  if (step > Lc) return;
  // the block's plane of the state and of T2 lie in their arrays (checked builds)
  if (!in_bounds((long long)(z + 1) * E * E - 1, v.N, ch.err) ||
      !in_bounds((long long)(z + 1) * v.by * v.bx - 1, ch.t2_stride, ch.err))
    return;
  const bool first = step == 0, last = step == Lc;
  const bool fixed = (flags & XF_FIXED_MOMENTUM) != 0;
  const bool need_q = !(first && !fixed);
  const int acc = st.acc;
  const long long N = v.N;
  const int bx = v.bx, by = v.by;
  const int tid = threadIdx.x;
  float2* Ub = ch.U + (long long)c * 2 * N;
  const float2* Usrc = Ub + (long long)(first ? acc : (acc ^ 1)) * N + (long long)z * E * E;
  float2* Udst = Ub + (long long)(acc ^ 1) * N + (long long)z * E * E;
  float2* Qc = ch.Q + (long long)c * N + (long long)z * E * E;
  const float* Sg = v.sinv + (long long)z * E * E;
  float2* T = ch.T2 + (long long)c * ch.t2_stride + (long long)z * by * bx;
  // the twiddles of length E in shared memory: the row and column stages load a lane's twiddles again for every
  // line, and as global loads (L1 hits) they were most of the kernel's load instructions (146.8 -> 140.9 us for
  // 64^2 planes x 64 chains)
  __shared__ float2 twE[E];
  for (int i = tid; i < E; i += NT) twE[i] = tw[tw_offset(E) + i];
  const float2* srcU = Usrc;
  const float2* srcQ = Qc;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw);
  if (!PREFETCH && (flags & XF_L2_PREFETCH) && tid == 0) {
    bulk_prefetch_l2(Usrc, E * E * 8);
    if (need_q) bulk_prefetch_l2(Qc, E * E * 8);
    bulk_prefetch_l2(Sg, E * E * 4);
  }
  if constexpr (PREFETCH) {
    // U and q only: 1/lambda is one array shared by every chain and stays in L2
    srcU = reinterpret_cast<const float2*>(smraw + Ly.u_off);
    srcQ = reinterpret_cast<const float2*>(smraw + Ly.q_off);
    if (tid == 0) {
      mbar_init(bar, 1);
      mbar_fence_init();
      const uint32_t bu = E * E * 8;
      mbar_arrive_expect_tx(bar, need_q ? 2 * bu : bu);
      bulk_g2s(smraw + Ly.u_off, Usrc, bu, bar);
      if (need_q) bulk_g2s(smraw + Ly.q_off, Qc, bu, bar);
    }
  }
  plane_load_box<E, NT>(sm, T, bx, by);
  __syncthreads();
  plane_fft<E>(sm, bx, by, +1, twE);
  if constexpr (PREFETCH) {
    const bool ok = mbar_wait_bounded(bar, 0);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(ch.err, 1);
        mbar_wait_bounded(bar, 0, 500000000ull);
      }
      return;
    }
  }
  double pa, pb;
  plane_update<E, NT, !PREFETCH>(sm, v, ch, st, c, z, first, last, need_q, flags, srcU, srcQ, Sg, Udst, Qc, pa, pb);
  plane_finish<E, NT>(sm, ch, c, z, first, last, pa, pb, T, bx, by, twE, red);
}

// ----------------------------------------------------------------- kriging products
// Chain-minor operands: X[j * Cp + c].  A warp's lanes are CG chain lanes x
// G = 32 / CG nonzero groups; each lane owns NR chains (c = cc + CG r).
//
// Batches of 32 nonzeros whose values and columns a warp loads before using any (csr_batches): 8 for 2-8 chains
// per warp (four chains on a 256x256x128 embedding: W 263 -> 235 us), 2 for one chain (deeper was slower there:
// 12.5 against 10.2 us on a 32^3 volume) and for 16, 1 for 32 (their gathers already overlap).
__host__ __device__ constexpr int csr_prefetch(int CG) { return (CG >= 2 && CG <= 8) ? 8 : (CG == 32 ? 1 : 2); }

// Accumulates sum_k val[k] X[col[k]] over the 32-nonzero batches b0, b0 + bs,
// ... of [ks, ke): the batch's values and columns are loaded once, coalesced,
// and broadcast by shuffle, so the X loads of a batch are independent and
// stay in flight together.
// n_cols bounds the column indices (checked builds; err receives the failure).
template <int CG, int NR, int PF>
__device__ __forceinline__ void csr_batches(const float* __restrict__ val, const int* __restrict__ col, int ks, int ke,
                                            int b0, int bs, const float* const (&x)[NR], int Cp, int lane,
                                            float (&acc)[NR], int n_cols, int* err) {
  constexpr int G = 32 / CG;
  const int grp = lane / CG;
  if constexpr (PF == 1) {
    for (int base = ks + b0 * 32; base < ke; base += bs * 32) {
      const int n = min(32, ke - base);
      const float mv = lane < n ? __ldg(val + base + lane) : 0.f;
      const int mc = lane < n ? __ldg(col + base + lane) : 0;
#pragma unroll
      for (int j0 = 0; j0 < 32; j0 += G) {
        const int j = j0 + grp;
        const float w = __shfl_sync(0xffffffffu, mv, j);
        const int cj = __shfl_sync(0xffffffffu, mc, j);
        const long long cidx = (long long)cj * Cp;
        if (j < n && in_bounds(cj, n_cols, err)) {
#pragma unroll
          for (int r = 0; r < NR; r++) acc[r] = fmaf(w, x[r][cidx], acc[r]);
        }
      }
    }
  } else {
    // PF batches of values and columns are loaded before any is used, so that several 256-byte loads per warp
    // are in flight while the matrix streams from memory; the batches are then consumed in their usual order.
    for (int base = ks + b0 * 32; base < ke; base += PF * bs * 32) {
      float mvp[PF];
      int mcp[PF], np[PF];
#pragma unroll
      for (int p = 0; p < PF; p++) {
        const int bb = base + p * bs * 32;
        np[p] = max(0, min(32, ke - bb));
        mvp[p] = lane < np[p] ? __ldg(val + bb + lane) : 0.f;
        mcp[p] = lane < np[p] ? __ldg(col + bb + lane) : 0;
      }
#pragma unroll
      for (int p = 0; p < PF; p++) {
        const int n = np[p];
        if (n == 0) break;
        const float mv = mvp[p];
        const int mc = mcp[p];
#pragma unroll
        for (int j0 = 0; j0 < 32; j0 += G) {
          const int j = j0 + grp;
          const float w = __shfl_sync(0xffffffffu, mv, j);
          const int cj = __shfl_sync(0xffffffffu, mc, j);
          const long long cidx = (long long)cj * Cp;
          if (j < n && in_bounds(cj, n_cols, err)) {
#pragma unroll
            for (int r = 0; r < NR; r++) acc[r] = fmaf(w, x[r][cidx], acc[r]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < NR; r++)
#pragma unroll
    for (int off = CG; off < 32; off <<= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], off);
}

// rs = Ys - W mu_D for every chain (MultiResParameters.h:361-363, 505-507),
// one block per row of W (grid-stride over rows); the 8 warps share the
// row's 32-nonzero batches and combine their sums in a fixed order.
template <int CG, int NR>
__global__ void __launch_bounds__(256, 4) k_spmv_w(DevVolume v, DevChains ch, int step, int sel, int chain_only) {
  grid_dep_wait();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int C = ch.C, Cp = ch.Cp;
  const int cc = lane % CG;
  __shared__ float red[8][CG * NR];
  const float* x[NR];
#pragma unroll
  for (int r = 0; r < NR; r++) {
    const int c = min(cc + CG * r, C - 1);
    x[r] = ch.muD + (long long)(ch.st[c].acc ^ sel) * v.n_h * Cp + c;
  }
  // thread t < C owns chain t for the row sums
  const int t = threadIdx.x;
  bool tact = false;
  if (t < C && (chain_only < 0 || t == chain_only)) tact = step < 0 || step <= ch.st[t].L_cur;
  double sq = 0.0;
  for (int row = blockIdx.x; row < v.n_s; row += gridDim.x) {
    float acc[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) acc[r] = 0.f;
    // batches ahead keep the matrix stream in flight (csr_prefetch)
    csr_batches<CG, NR, csr_prefetch(CG)>(v.w_val, v.w_col, v.w_rowptr[row], v.w_rowptr[row + 1], warp, 8, x, Cp,
                                          lane, acc, v.n_h, ch.err);
    if (lane < CG) {
#pragma unroll
      for (int r = 0; r < NR; r++) red[warp][lane + CG * r] = acc[r];
    }
    __syncthreads();
    if (tact) {
      float s = 0.f;
#pragma unroll
      for (int w = 0; w < 8; w++) s += red[w][t];
      const float rsv = v.Ys[row] - s;
      ch.rs[(long long)row * Cp + t] = rsv;
      sq += (double)rsv * rsv;
    }
    __syncthreads();
  }
  if (tact) {
    const int slot = step <= 0 ? SL_RS0 : (step == ch.st[t].L_cur ? SL_RSL : SL_SCRATCH);
    ch.part[((long long)t * NSLOT + slot) * ch.maxblk + blockIdx.x] = sq;
  }
}

// The same product with one warp per row of W (grid-stride over rows by warps), for kriging matrices with many
// rows per block (large volumes with few chains): no block barrier per row, and every warp keeps 8 batches of its
// row in flight.  The per-chain squared residuals are summed over the block's warps in a fixed order.
template <int CG, int NR>
__global__ void __launch_bounds__(256, 4) k_spmv_w_rows(DevVolume v, DevChains ch, int step, int sel, int chain_only) {
  grid_dep_wait();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int C = ch.C, Cp = ch.Cp;
  const int cc = lane % CG;
  __shared__ double red[8][CG * NR];
  bool act[NR];
  double sq[NR];
  const float* x[NR];
#pragma unroll
  for (int r = 0; r < NR; r++) {
    const int c = cc + CG * r;
    const int cs = min(c, C - 1);
    x[r] = ch.muD + (long long)(ch.st[cs].acc ^ sel) * v.n_h * Cp + cs;
    act[r] = false;
    sq[r] = 0.0;
    if (c < C && (chain_only < 0 || c == chain_only)) act[r] = step < 0 || step <= ch.st[c].L_cur;
  }
  for (int row = blockIdx.x * 8 + warp; row < v.n_s; row += gridDim.x * 8) {
    float acc[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) acc[r] = 0.f;
    csr_batches<CG, NR, 8>(v.w_val, v.w_col, v.w_rowptr[row], v.w_rowptr[row + 1], 0, 1, x, Cp, lane, acc, v.n_h,
                           ch.err);
    if (lane < CG) {
      const float ys = v.Ys[row];
#pragma unroll
      for (int r = 0; r < NR; r++) {
        if (!act[r]) continue;
        const float rsv = ys - acc[r];
        ch.rs[(long long)row * Cp + cc + CG * r] = rsv;
        sq[r] += (double)rsv * rsv;
      }
    }
  }
  if (lane < CG) {
#pragma unroll
    for (int r = 0; r < NR; r++) red[warp][lane + CG * r] = sq[r];
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    if (chain_only >= 0 && c != chain_only) continue;
    const ChainState& st = ch.st[c];
    if (step >= 0 && step > st.L_cur) continue;
    double t = 0.0;
    for (int w = 0; w < 8; w++) t += red[w][c];
    const int slot = step <= 0 ? SL_RS0 : (step == st.L_cur ? SL_RSL : SL_SCRATCH);
    ch.part[((long long)c * NSLOT + slot) * ch.maxblk + blockIdx.x] = t;
  }
}

// gD = sigma_h^-2 (Yh - mu_D) + sigma_s^-2 W^T rs (MultiResParameters.h:357-364),
// one warp per data voxel over the transposed CSR (grid-stride), plus the
// ||Yh - mu_D||^2 partials per block.
template <int CG, int NR>
__global__ void __launch_bounds__(256, 4) k_spmv_wt(DevVolume v, DevChains ch, int step, int sel, int chain_only) {
  grid_dep_wait();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int C = ch.C, Cp = ch.Cp;
  const int cc = lane % CG;
  __shared__ double red[8][CG * NR];
  bool act[NR];
  double sq[NR];
  int half[NR];
  float shv[NR], ssv[NR];
  const float* x[NR];
#pragma unroll
  for (int r = 0; r < NR; r++) {
    const int c = cc + CG * r;
    const int cs = min(c, C - 1);
    x[r] = ch.rs + cs;
    act[r] = false;
    sq[r] = 0.0;
    half[r] = 0;
    shv[r] = ssv[r] = 0.f;
    if (c < C && (chain_only < 0 || c == chain_only)) {
      const ChainState& st = ch.st[c];
      act[r] = step < 0 || step <= st.L_cur;
      half[r] = st.acc ^ sel;
      shv[r] = st.sh;
      ssv[r] = st.ss;
    }
  }
  for (int row = blockIdx.x * 8 + warp; row < v.n_h; row += gridDim.x * 8) {
    float acc[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) acc[r] = 0.f;
    if (v.n_s > 0)
      csr_batches<CG, NR, csr_prefetch(CG) < 2 ? 2 : csr_prefetch(CG)>(v.wt_val, v.wt_col, v.wt_rowptr[row],
                                                                       v.wt_rowptr[row + 1], 0, 1, x, Cp, lane, acc,
                                                                       v.n_s, ch.err);
    if (lane < CG) {
      const float yh = v.Yh[row];
#pragma unroll
      for (int r = 0; r < NR; r++) {
        if (!act[r]) continue;
        const int c = cc + CG * r;
        const float m = ch.muD[((long long)half[r] * v.n_h + row) * Cp + c];
        const float rh = yh - m;
        ch.gD[(long long)row * Cp + c] = shv[r] * rh + ssv[r] * acc[r];
        sq[r] += (double)rh * rh;
      }
    }
  }
  if (lane < CG) {
#pragma unroll
    for (int r = 0; r < NR; r++) red[warp][lane + CG * r] = sq[r];
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    if (chain_only >= 0 && c != chain_only) continue;
    const ChainState& st = ch.st[c];
    if (step >= 0 && step > st.L_cur) continue;
    double s = 0.0;
    for (int w = 0; w < 8; w++) s += red[w][c];
    const int slot = step <= 0 ? SL_RH0 : (step == st.L_cur ? SL_RHL : SL_SCRATCH);
    ch.part[((long long)c * NSLOT + slot) * ch.maxblk + blockIdx.x] = s;
  }
}

// ----------------------------------------------------------------- per-iteration scalars
// The arguments of MultiResParameters::update: eps() and integrator_steps()
// (gaussian_process_model.h:135).
__global__ void k_iter_begin(DevChains ch) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ch.C) return;
  ChainState& st = ch.st[c];
  if (st.done) {
    st.L_cur = -1;
    return;
  }
  const u32x4 r = philox(u32x4{0u, (uint32_t)st.iteration, (uint32_t)(ch.chain0 + c), RNG_SCALAR}, ch.seed);
  st.eps_cur = hmc_eps(st, u01d(r.x, r.y));
  st.L_cur = hmc_steps(st);
}

__device__ double slot_sum(const DevChains& ch, int c, int slot, int nb, double* red) {
  double s = 0.0;
  const double* p = ch.part + ((long long)c * NSLOT + slot) * ch.maxblk;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) s += p[i];
  return block_sum(s, red);
}

// Metropolis accept (MultiResParameters.h:702-726), Gibbs sigma draws
// (:821-838) and HMCParameters::update (HMCParameters.h:259-297).  The
// Hamiltonian difference is formed in FP64.
__global__ void __launch_bounds__(256) k_accept(DevVolume v, DevChains ch) {
  __shared__ double red[8];
  __shared__ double sums[8];
  const int c = blockIdx.x;
  ChainState& st = ch.st[c];
  if (st.L_cur < 0) return;
  const int nbs[8] = {ch.nb_x, ch.nb_x, ch.nb_wt, ch.nb_w, ch.nb_x, ch.nb_x, ch.nb_wt, ch.nb_w};
  for (int s = 0; s < 8; s++) {
    double t = 0.0;
    if (!((s == SL_RS0 || s == SL_RSL) && v.n_s == 0)) t = slot_sum(ch, c, s, nbs[s], red);
    if (threadIdx.x == 0) sums[s] = t;
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double N = (double)v.N;
  const double sh = st.sh, ss = st.ss;
  const double lp0 = -0.5 * sums[SL_LP0] / N;
  const double ll0 = -0.5 * (sh * sums[SL_RH0] + (v.n_s > 0 ? ss * sums[SL_RS0] : 0.0));
  const double E0 = -0.5 * sums[SL_E0] + lp0 + ll0;
  const double lpL = -0.5 * sums[SL_LPL] / N;
  const double llL = -0.5 * (sh * sums[SL_RHL] + (v.n_s > 0 ? ss * sums[SL_RSL] : 0.0));
  const double KL = -0.5 * sums[SL_KL] / N;
  const double logR = (lpL + llL + KL) - E0;
  double R = exp(logR);
  if (isnan(R)) R = 0.0;
  const u32x4 r = philox(u32x4{0u, (uint32_t)st.iteration, (uint32_t)(ch.chain0 + c), RNG_SCALAR}, ch.seed);
  const double u = u01d(r.z, r.w);
  double Rh = sums[SL_RH0], Rs = sums[SL_RS0];
  if (u < R) {
    st.acc ^= 1;
    st.accepted += 1;
    Rh = sums[SL_RHL];
    Rs = sums[SL_RSL];
  }
  st.Rh_acc = Rh;
  st.Rs_acc = Rs;
  // Gibbs: shape n/2 + 1, rate ||residual||^2 / 2 (float arithmetic as in the reference)
  const float shape_h = 0.5f * (float)v.n_h + 1.0f, rate_h = 0.5f * (float)Rh;
  st.sh = (float)gamma_draw(shape_h, 1.0 / (double)rate_h, ch.seed, RNG_SCALAR, ch.chain0 + c, st.iteration, 16u, &st.err);
  if (v.n_s > 0) {
    const float shape_s = 0.5f * (float)v.n_s + 1.0f, rate_s = 0.5f * (float)Rs;
    st.ss = (float)gamma_draw(shape_s, 1.0 / (double)rate_s, ch.seed, RNG_SCALAR, ch.chain0 + c, st.iteration, 4096u,
                              &st.err);
  }
  st.grad_evals += st.L_cur + 1;
  st.last_log_ratio = logR;
  st.last_E0 = E0;
  st.last_Ep = lpL + llL + KL;
  hmc_update(st, (float)fmin(1.0, R));
  st.save_now = 0;
  if (hmc_save_iteration(st)) {
    st.save_now = 1;
    st.saved += 1;
    const double ll = -0.5 * ((double)st.sh * Rh + (v.n_s > 0 ? (double)st.ss * Rs : 0.0));
    st.ll_sum += ll;
    st.sigh_sum += sqrt(1.0 / (double)st.sh);
    st.sigs_sum += v.n_s > 0 ? sqrt(1.0 / (double)st.ss) : 0.0;
    if (ch.save_rec != nullptr && st.saved <= st.n_save) {
      // MultiResParameters::sigma (MultiResParameters.h:613-619) is sqrt(1 / sigma^-2) in float
      double* r = ch.save_rec + ((long long)(st.saved - 1) * ch.C + c) * 3;
      r[0] = (double)sqrtf(1.0f / st.sh);
      r[1] = v.n_s > 0 ? (double)sqrtf(1.0f / st.ss) : 0.0;
      r[2] = ll;
    }
    if (st.saved >= st.n_save) st.done = 1;
  }
}

// mcmc_summary::update (gaussian_process_model.h:209-229): max |mu| per chain, then moments.
__global__ void __launch_bounds__(256) k_summary_max(DevVolume v, DevChains ch) {
  __shared__ float red[8];
  const int c = blockIdx.x;
  ChainState& st = ch.st[c];
  if (!st.save_now || st.L_cur < 0) return;
  const float* mo = ch.muO + (long long)st.acc * v.n_o * ch.Cp + c;
  float m = 0.f;
  for (int o = threadIdx.x; o < v.n_o; o += blockDim.x) m = fmaxf(m, fabsf(mo[(long long)o * ch.Cp]));
  for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); i++) m = fmaxf(m, red[i]);
    m = fmaxf(m, red[0]);
    st.maxabs = m;
  }
}

__global__ void k_summary_acc(DevVolume v, DevChains ch) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)v.n_o * ch.Cp;
  if (e >= total) return;
  const int c = (int)(e % ch.Cp);
  if (c >= ch.C) return;
  const ChainState& st = ch.st[c];
  if (!st.save_now || st.L_cur < 0) return;
  const float val = ch.muO[(long long)st.acc * v.n_o * ch.Cp + e];
  ch.s1[e] += val;
  ch.s2[e] += (double)val * val;
  ch.sa[e] += fabs((double)val) / fmax((double)st.maxabs, 1e-6);
  if (ch.samples != nullptr) ch.samples[(long long)(st.saved - 1) * total + e] = val;
}

// ----------------------------------------------------------------- initialisation
// _initialize_sigma (MultiResParameters.h:764-778): sigma_h^-2 ~ Gamma(v, 1),
// sigma_s^-2 = sigma_h^-2 / U(0, 1).
__global__ void k_init_sigma(DevChains ch, float shape, int n_datasets) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ch.C) return;
  ChainState& st = ch.st[c];
  st.sh = (float)gamma_draw((double)shape, 1.0, ch.seed, RNG_INIT_SIGMA, ch.chain0 + c, 0u, 16u, &st.err);
  const u32x4 r = philox(u32x4{0u, 0u, (uint32_t)(ch.chain0 + c), RNG_INIT_SIGMA}, ch.seed);
  st.ss = n_datasets == 2 ? st.sh / u01f(r.x) : 1.0f;
}

// gD <- Yh for all chains (the data part of the initial state, add_data_to_mu).
__global__ void k_fill_gD(DevVolume v, DevChains ch) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)v.n_h * ch.Cp) return;
  ch.gD[e] = v.Yh[e / ch.Cp];
}

// _initialize_mu (MultiResParameters.h:744-759) in the spectral basis:
// u0 += sqrt(N lambda) w / 10 on live modes, w ~ CN(0, 2).
__global__ void k_init_prior(DevVolume v, DevChains ch) {
  const long long pair = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (2 * pair >= v.N) return;
  const long long gi = 2 * pair;
  float2* U = ch.U + (long long)c * 2 * v.N + (long long)ch.st[c].acc * v.N;
  const u32x4 r = philox(u32x4{(uint32_t)pair, 0u, (uint32_t)(ch.chain0 + c), RNG_INIT_MU}, ch.seed);
  const float2 w0 = box_muller(u01f(r.x), u01f(r.y)), w1 = box_muller(u01f(r.z), u01f(r.w));
  const float Nf = (float)v.N;
#pragma unroll
  for (int m = 0; m < 2; m++) {
    const float s = v.sinv[gi + m];
    if (s > 0.0f) {
      const float a = sqrtf(Nf / s) * 0.1f;
      const float2 w = m == 0 ? w0 : w1;
      U[gi + m].x += a * w.x;
      U[gi + m].y += a * w.y;
    }
  }
}

// ----------------------------------------------------------------- spectrum (FP64, one-time)
// circulant_base_3d (circulant_base.inl:30-89): wrapped offsets, float norm of
// Q (o, 0), covariance evaluated in FP64.
__global__ void k_base(double2* base, int E0, int E1, int E2, float q00, float q01, float q02, float q10, float q11,
                       float q12, float q20, float q21, float q22, double th0, double th1, double th2, int covfun) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long N = (long long)E0 * E1 * E2;
  if (i >= N) return;
  const int l = (int)(i % E0), m = (int)((i / E0) % E1), n = (int)(i / ((long long)E0 * E1));
  const float o0 = (float)(l <= E0 / 2 ? l : E0 - l), o1 = (float)(m <= E1 / 2 ? m : E1 - m),
              o2 = (float)(n <= E2 / 2 ? n : E2 - n);
  // float arithmetic in source order with every product and sum rounded (no fused multiply-add), so the
  // distances equal a plain float evaluation of the same expression on the host
  const float a = __fadd_rn(__fadd_rn(__fmul_rn(q00, o0), __fmul_rn(q01, o1)), __fmul_rn(q02, o2));
  const float b = __fadd_rn(__fadd_rn(__fmul_rn(q10, o0), __fmul_rn(q11, o1)), __fmul_rn(q12, o2));
  const float cc = __fadd_rn(__fadd_rn(__fmul_rn(q20, o0), __fmul_rn(q21, o1)), __fmul_rn(q22, o2));
  const double d = (double)__fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)), __fmul_rn(cc, cc)));
  double val;
  if (covfun == 0)
    val = th0 * exp(-th1 * pow(fabs(d), th2));
  else
    val = th0 * pow(1.0 + th1 / th2 * d * d, -th2);
  base[i] = make_double2(val, 0.0);
}

// S = {Re lambda <= 0} (MultiResParameters.h:258-262); sinv = 1/Re lambda on live modes.
__global__ void k_spectrum(const double2* lam, float* sinv, double* lam_re, long long N, int* n_S) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double re = lam[i].x;
  lam_re[i] = re;
  if (re > 0.0) {
    sinv[i] = (float)(1.0 / re);
  } else {
    sinv[i] = -1.0f;
    atomicAdd(n_S, 1);
  }
}

// ----------------------------------------------------------------- evaluation helpers
// Re field[idx[j]] for j < n; N bounds the indices (checked builds, failures to err).
__global__ void k_gather_re(const float2* field, const int* idx, int n, float* out, int pitch, int col, long long N,
                            int* err) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n && in_bounds(idx[j], N, err)) out[(long long)j * pitch + col] = field[idx[j]].x;
}

// Block partials of sum_live |u|^2 * sinv  (mode 0) or sum_live |u|^2 / (sinv + sh)  (mode 1).
__global__ void __launch_bounds__(256) k_spectral_energy(const float2* u, const float* sinv, long long N, float sh,
                                                         int mode, double* part) {
  __shared__ double red[8];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const float s = sinv[i];
    if (s > 0.f) {
      const double m2 = (double)u[i].x * u[i].x + (double)u[i].y * u[i].y;
      acc += mode == 0 ? m2 * s : m2 / (double)(s + sh);
    }
  }
  const double t = block_sum(acc, red);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_scale(float2* u, long long N, float f) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) u[i] = make_float2(u[i].x * f, u[i].y * f);
}

// Device restatement of HMCParameters::update over a given MH-rate sequence (diagnostics).
// A wait that runs out: an mbarrier that nothing arrives on, waited for with a limit of limit_ms (the bounded-wait
// path every pipeline in this library takes when a copy or an MMA does not complete).
__global__ void k_debug_bounded_wait(uint64_t limit_ns, int* gave_up, unsigned long long* waited_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  mbar_fence_init();
  const uint64_t t0 = globaltimer_ns();
  const bool ok = mbar_wait_bounded(&bar, 0, limit_ns);
  *waited_ns = globaltimer_ns() - t0;
  *gave_up = ok ? 0 : 1;
}

__global__ void k_debug_dual_averaging(ChainState st, int n, const float* rates, double* eps_out, int* steps_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int i = 0; i < n; i++) {
    hmc_update(st, rates[i]);
    eps_out[i] = st.eps;
    steps_out[i] = hmc_steps(st);
  }
}

}  // namespace drb
