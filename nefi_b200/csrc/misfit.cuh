// Fused trace misfit: residual -> zero-phase low-pass -> masked mean square -> adjoint source, in one
// pass over the traces (nefi/instances/wave_fwi/losses.py:38-86 `lowpass` / `BandLimitedMSE`, and the
// sensor response of nefi/instances/photoacoustic3d/sensor.py:24-66 `gaussian_lowpass`).
//
// Each filter of the reference is a real, even frequency response applied to a zero-padded trace and
// cropped back to n samples; on [0, n) that is a linear convolution with lags in (-n, n). Any FFT length
// L >= 2n evaluates it exactly, so the kernels use L = 2^k with the response re-sampled on the host
// (float64) from the reference's own window: the device receives Hp[p] = H_L[bitrev(p)] / L.
//
// One CTA owns two traces at a time (re = trace 2j, im = trace 2j+1: a real, even response keeps them
// apart), held in shared memory as L complex values. A filter is a decimation-in-frequency FFT (natural
// order in, bit-reversed out), a multiply by Hp, and a decimation-in-time inverse FFT (bit-reversed in,
// natural out): no permutation pass. Stages run four at a time in registers (radix-16 groups); the top
// group of an inverse FFT and of the next forward FFT touch the same indices, so the pointwise work
// between two filters (subtract the observation, square and mask, crop to n) happens in registers
// inside that merged pass. Global memory is touched once per trace for each input and output.
#pragma once

#include <cstdint>

namespace nw {
namespace fft {

template <typename T> struct Cx;
template <> struct Cx<float> { using t = float2; };
template <> struct Cx<double> { using t = double2; };

template <typename T>
__device__ __forceinline__ typename Cx<T>::t cmul(typename Cx<T>::t a, typename Cx<T>::t b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
__device__ __forceinline__ typename Cx<T>::t cmulc(typename Cx<T>::t a, typename Cx<T>::t b) {  // a * conj(b)
  return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}

__device__ __forceinline__ void sincos_pi(float x, float* s, float* c) { sincospif(x, s, c); }
__device__ __forceinline__ void sincos_pi(double x, double* s, double* c) { sincospi(x, s, c); }

// shared-memory slot of element i: one pad slot every 16 elements spreads strided groups over banks
__host__ __device__ __forceinline__ int slot(int i) { return i + (i >> 4); }

// Stage groups, top (most significant bits) first: group j covers bits [sbit, sbit + nb).
struct Groups {
  int log2_len, count;
  int sbit[8], nb[8], tab_off[16];  // tab_off[t]: offset of stage t's twiddles W_{2^{t+1}}^l, l < 2^sbit
  int tab_len;
};

__host__ __device__ inline Groups make_groups(int log2_len) {
  Groups g{};
  g.log2_len = log2_len;
  g.count = 0;
  for (int hi = log2_len; hi > 0;) {
    const int nb = hi >= 4 ? 4 : hi;
    g.sbit[g.count] = hi - nb;
    g.nb[g.count] = nb;
    ++g.count;
    hi -= nb;
  }
  int off = 16;  // the first 16 entries hold W_16^j, j < 8 (the in-group factors), padded
  for (int t = 0; t < log2_len; ++t) {
    int sb = 0;
    for (int j = 0; j < g.count; ++j)
      if (t >= g.sbit[j] && t < g.sbit[j] + g.nb[j]) sb = g.sbit[j];
    g.tab_off[t] = off;
    off += 1 << sb;
  }
  g.tab_len = off;
  return g;
}

// Twiddle tables: tab[j] = W_16^j (j < 8); stage t: tab[tab_off[t] + l] = W_{2^{t+1}}^l = exp(-2 pi i l / 2^{t+1}).
template <typename T>
__device__ void build_tables(const Groups& G, typename Cx<T>::t* tab) {
  for (int j = threadIdx.x; j < 8; j += blockDim.x) {
    T s, c;
    sincos_pi(-(T)j / (T)8, &s, &c);
    tab[j] = {c, s};
  }
  for (int t = 0; t < G.log2_len; ++t) {
    const int n = (t + 1 < G.log2_len ? G.tab_off[t + 1] : G.tab_len) - G.tab_off[t];
    for (int l = threadIdx.x; l < n; l += blockDim.x) {
      T s, c;
      sincos_pi(-(T)l / (T)(1 << t), &s, &c);  // exact argument: l / 2^t
      tab[G.tab_off[t] + l] = {c, s};
    }
  }
}

// Forward (DIF) stages of one group held in v[0..2^NB): stage t = sbit + u for u = NB-1 .. 0.
template <typename T, int NB>
__device__ __forceinline__ void dif_group(typename Cx<T>::t* v, int low, int sbit, const Groups& G,
                                          const typename Cx<T>::t* tab) {
  using C = typename Cx<T>::t;
#pragma unroll
  for (int u = NB - 1; u >= 0; --u) {
    const int half = 1 << u;
    const C wl = tab[G.tab_off[sbit + u] + low];
#pragma unroll
    for (int k = 0; k < (1 << NB); ++k) {
      if (k & half) continue;
      const C a = v[k], b = v[k + half];
      v[k] = {a.x + b.x, a.y + b.y};
      const C d = {a.x - b.x, a.y - b.y};
      const int j = k & (half - 1);
      C w = wl;
      if (j) w = cmul<T>(wl, tab[j << (3 - u)]);
      v[k + half] = cmul<T>(d, w);
    }
  }
}

// Inverse (DIT, conjugate twiddles) stages of one group: stage t = sbit + u for u = 0 .. NB-1.
template <typename T, int NB>
__device__ __forceinline__ void dit_group(typename Cx<T>::t* v, int low, int sbit, const Groups& G,
                                          const typename Cx<T>::t* tab) {
  using C = typename Cx<T>::t;
#pragma unroll
  for (int u = 0; u < NB; ++u) {
    const int half = 1 << u;
    const C wl = tab[G.tab_off[sbit + u] + low];
#pragma unroll
    for (int k = 0; k < (1 << NB); ++k) {
      if (k & half) continue;
      const int j = k & (half - 1);
      C w = wl;
      if (j) w = cmul<T>(wl, tab[j << (3 - u)]);
      const C a = v[k];
      const C b = cmulc<T>(v[k + half], w);
      v[k] = {a.x + b.x, a.y + b.y};
      v[k + half] = {a.x - b.x, a.y - b.y};
    }
  }
}

}  // namespace fft

using fft::Cx;

// ------------------------------------------------------------------------------------------------
// the fused program
// ------------------------------------------------------------------------------------------------
enum : unsigned {
  MF_LOAD_PRED = 1u,  // x = pred
  MF_LOAD_OBS = 2u,   // x = obs
  MF_SUB_OBS = 4u,    // x -= obs
  MF_LOSS = 8u,       // sum += m x^2, count += m, x = m x
  MF_STORE = 16u,     // grad = scale x (ends the program)
  MF_END = 32u,       // ends the program
};

// slots of the caller's state array (doubles) after the per-CTA partial sums
constexpr int kMisfitCtas = 1024;
constexpr int kStCount = 2 * kMisfitCtas, kStDen = kStCount + 1, kStScale = kStCount + 2, kStNum = kStCount + 3,
              kStLoss = kStCount + 4, kStInv = kStCount + 5, kStateLen = kStCount + 8;

template <typename T>
struct MisfitArgs {
  const T* pred;
  const T* obs;
  const T* mask;  // NULL, per trace or per sample
  const T* spec[4];  // bit-reversed responses / L, one per filter
  T* grad;
  const double* state;  // gradient scale for MF_STORE (NULL: 1)
  double* partials;     // 2 per CTA: sum, count (NULL: not wanted)
  long long n_traces;
  int n_t, mask_per_sample, n_filters;
  unsigned op[5];  // op[0] before the first filter, op[f + 1] after filter f
};

template <typename T>
struct PairCtx {  // the two traces a CTA holds
  long long ta, tb;  // tb < 0: no second trace
  T ma, mb;          // per-trace mask values (1 without a mask)
};

template <typename T>
__device__ __forceinline__ T mask_at(const MisfitArgs<T>& a, long long tr, int i, T per_trace) {
  return (a.mask && a.mask_per_sample) ? a.mask[tr * a.n_t + i] : per_trace;
}

// Pointwise work at sample i of both traces: x = (re, im) after a filter (or zero before the first).
template <typename T>
__device__ __forceinline__ void apply_op(const MisfitArgs<T>& a, const PairCtx<T>& pc, unsigned op, int i,
                                         typename Cx<T>::t& x, double& acc, double& cnt, T scale) {
  if (i >= a.n_t) {  // crop: the convolution's tail beyond the trace is not part of the result
    x = {(T)0, (T)0};
    return;
  }
  const bool has_b = pc.tb >= 0;
  const long long ia = pc.ta * a.n_t + i, ib = pc.tb * a.n_t + i;
  if (op & MF_LOAD_PRED) x = {a.pred[ia], has_b ? a.pred[ib] : (T)0};
  if (op & MF_LOAD_OBS) x = {a.obs[ia], has_b ? a.obs[ib] : (T)0};
  if (op & MF_SUB_OBS) {
    x.x -= a.obs[ia];
    if (has_b) x.y -= a.obs[ib];
  }
  if (op & MF_LOSS) {
    const T ma = mask_at(a, pc.ta, i, pc.ma);
    const T mb = has_b ? mask_at(a, pc.tb, i, pc.mb) : (T)0;
    acc += (double)(ma * x.x * x.x) + (double)(mb * x.y * x.y);
    cnt += (double)ma + (double)mb;
    x = {ma * x.x, mb * x.y};
  }
  if (op & MF_STORE) {
    a.grad[ia] = scale * x.x;
    if (has_b) a.grad[ib] = scale * x.y;
  }
}

template <typename T, int NB>
__device__ __forceinline__ void load_group(const typename Cx<T>::t* s, typename Cx<T>::t* v, int base, int sbit) {
#pragma unroll
  for (int k = 0; k < (1 << NB); ++k) v[k] = s[fft::slot(base + (k << sbit))];
}
template <typename T, int NB>
__device__ __forceinline__ void store_group(typename Cx<T>::t* s, const typename Cx<T>::t* v, int base, int sbit) {
#pragma unroll
  for (int k = 0; k < (1 << NB); ++k) s[fft::slot(base + (k << sbit))] = v[k];
}

// One pass of group j (not the top one, not the last one) over all groups: DIF or DIT.
template <typename T, bool DIF>
__device__ __forceinline__ void inner_pass(typename Cx<T>::t* s, const fft::Groups& G, int j,
                                           const typename Cx<T>::t* tab) {
  const int sbit = G.sbit[j];
  const int n_groups = 1 << (G.log2_len - 4);
  for (int gi = threadIdx.x; gi < n_groups; gi += blockDim.x) {
    const int low = gi & ((1 << sbit) - 1);
    const int base = ((gi >> sbit) << (sbit + 4)) | low;
    typename Cx<T>::t v[16];
    load_group<T, 4>(s, v, base, sbit);
    if (DIF) fft::dif_group<T, 4>(v, low, sbit, G, tab);
    else fft::dit_group<T, 4>(v, low, sbit, G, tab);
    store_group<T, 4>(s, v, base, sbit);
  }
}

// The 2^NB response values of one lowest group: contiguous and aligned to their size, so they are read
// as 16-byte vectors where they fill one (the response stays in L2; every CTA re-reads it per pair).
template <typename T, int NB>
__device__ __forceinline__ void load_response(const T* __restrict__ src, T* h) {
  constexpr int kBytes = (1 << NB) * (int)sizeof(T);
  if constexpr (kBytes >= 16) {
#pragma unroll
    for (int c = 0; c < kBytes / 16; ++c) {
      const float4 q = __ldg(reinterpret_cast<const float4*>(src) + c);
      memcpy(reinterpret_cast<char*>(h) + 16 * c, &q, 16);
    }
  } else {
#pragma unroll
    for (int k = 0; k < (1 << NB); ++k) h[k] = __ldg(src + k);
  }
}

// The lowest group (bits [0, NB)): forward stages, the response, inverse stages.
template <typename T, int NB>
__device__ __forceinline__ void middle_pass(typename Cx<T>::t* s, const fft::Groups& G, const T* __restrict__ spec,
                                            const typename Cx<T>::t* tab) {
  const int n_groups = 1 << (G.log2_len - NB);
  for (int gi = threadIdx.x; gi < n_groups; gi += blockDim.x) {
    const int base = gi << NB;
    typename Cx<T>::t v[1 << NB];
    load_group<T, NB>(s, v, base, 0);
    fft::dif_group<T, NB>(v, 0, 0, G, tab);
    T h[1 << NB];
    load_response<T, NB>(spec + base, h);
#pragma unroll
    for (int k = 0; k < (1 << NB); ++k) v[k] = {v[k].x * h[k], v[k].y * h[k]};
    fft::dit_group<T, NB>(v, 0, 0, G, tab);
    store_group<T, NB>(s, v, base, 0);
  }
}

// The top group (bits [log2 L - 4, log2 L)): optional inverse stages (the end of filter f), the pointwise op at the
// natural-order samples, optional forward stages (the start of filter f + 1).
template <typename T>
__device__ __forceinline__ void top_pass(typename Cx<T>::t* s, const fft::Groups& G, const MisfitArgs<T>& a,
                                         const PairCtx<T>& pc, bool inverse_first, unsigned op, bool forward_after,
                                         const typename Cx<T>::t* tab, double& acc, double& cnt, T scale) {
  const int sbit = G.sbit[0];
  const int n_groups = 1 << sbit;
  for (int gi = threadIdx.x; gi < n_groups; gi += blockDim.x) {
    typename Cx<T>::t v[16];
    if (inverse_first) {
      load_group<T, 4>(s, v, gi, sbit);
      fft::dit_group<T, 4>(v, gi, sbit, G, tab);
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = {(T)0, (T)0};
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) apply_op<T>(a, pc, op, gi + (k << sbit), v[k], acc, cnt, scale);
    if (forward_after) {
      fft::dif_group<T, 4>(v, gi, sbit, G, tab);
      store_group<T, 4>(s, v, gi, sbit);
    }
  }
}

template <typename T>
__device__ __forceinline__ void block_partials(double acc, double cnt, double* out) {
  __shared__ double red[2][32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc += __shfl_down_sync(0xffffffffu, acc, o);
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    red[0][w] = acc;
    red[1][w] = cnt;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    acc = l < nw ? red[0][l] : 0.0;
    cnt = l < nw ? red[1][l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      acc += __shfl_down_sync(0xffffffffu, acc, o);
      cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    if (l == 0 && out) {
      out[2 * blockIdx.x] = acc;
      out[2 * blockIdx.x + 1] = cnt;
    }
  }
}

template <typename T, int NB>
__device__ __forceinline__ void middle_dispatch_(typename Cx<T>::t* s, const fft::Groups& G, const T* spec,
                                                 const typename Cx<T>::t* tab) {
  middle_pass<T, NB>(s, G, spec, tab);
}

// Persistent CTAs over trace pairs; dynamic shared memory = twiddle tables + L padded complex slots.
template <typename T>
constexpr int misfit_threads() { return sizeof(T) == 8 ? 256 : 512; }  // float64 needs twice the registers

template <typename T>
__global__ void __launch_bounds__(misfit_threads<T>()) misfit_fft_kernel(MisfitArgs<T> a, fft::Groups Gp) {
  using C = typename Cx<T>::t;
  extern __shared__ __align__(16) unsigned char misfit_smem[];
  __shared__ fft::Groups G;
  if (threadIdx.x == 0) G = Gp;
  __syncthreads();
  C* tab = reinterpret_cast<C*>(misfit_smem);
  C* s = tab + G.tab_len;
  fft::build_tables<T>(G, tab);
  __syncthreads();
  bool stores = false;
  for (int f = 0; f <= a.n_filters; ++f) stores |= (a.op[f] & MF_STORE) != 0;
  const T scale = (stores && a.state) ? (T)a.state[kStScale] : (T)1;
  double acc = 0.0, cnt = 0.0;
  const long long n_pairs = (a.n_traces + 1) / 2;
  for (long long p = blockIdx.x; p < n_pairs; p += gridDim.x) {
    PairCtx<T> pc;
    pc.ta = 2 * p;
    pc.tb = 2 * p + 1 < a.n_traces ? 2 * p + 1 : -1;
    const bool per_trace = a.mask && !a.mask_per_sample;
    pc.ma = per_trace ? a.mask[pc.ta] : (T)1;
    pc.mb = (per_trace && pc.tb >= 0) ? a.mask[pc.tb] : (T)1;
    top_pass<T>(s, G, a, pc, false, a.op[0], true, tab, acc, cnt, scale);
    __syncthreads();
    for (int f = 0; f < a.n_filters; ++f) {
      for (int j = 1; j < G.count - 1; ++j) {
        inner_pass<T, true>(s, G, j, tab);
        __syncthreads();
      }
      switch (G.nb[G.count - 1]) {
        case 1: middle_dispatch_<T, 1>(s, G, a.spec[f], tab); break;
        case 2: middle_dispatch_<T, 2>(s, G, a.spec[f], tab); break;
        case 3: middle_dispatch_<T, 3>(s, G, a.spec[f], tab); break;
        default: middle_dispatch_<T, 4>(s, G, a.spec[f], tab); break;
      }
      __syncthreads();
      for (int j = G.count - 2; j >= 1; --j) {
        inner_pass<T, false>(s, G, j, tab);
        __syncthreads();
      }
      const unsigned op = a.op[f + 1];
      const bool more = f + 1 < a.n_filters && !(op & (MF_STORE | MF_END));
      top_pass<T>(s, G, a, pc, true, op, more, tab, acc, cnt, scale);
      __syncthreads();
      if (!more) break;
    }
  }
  block_partials<T>(acc, cnt, a.partials);
}

// The same program without filters: one grid-stride pass over the samples.
template <typename T>
__global__ void __launch_bounds__(256) misfit_plain_kernel(MisfitArgs<T> a) {
  const unsigned op = a.op[0];
  const T scale = ((op & MF_STORE) && a.state) ? (T)a.state[kStScale] : (T)1;
  double acc = 0.0, cnt = 0.0;
  const long long N = a.n_traces * a.n_t;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
    const long long tr = e / a.n_t;
    T x = (T)0;
    if (op & MF_LOAD_PRED) x = a.pred[e];
    if (op & MF_LOAD_OBS) x = a.obs[e];
    if (op & MF_SUB_OBS) x -= a.obs[e];
    if (op & MF_LOSS) {
      const T m = a.mask ? (a.mask_per_sample ? a.mask[e] : a.mask[tr]) : (T)1;
      acc += (double)(m * x * x);
      cnt += (double)m;
      x = m * x;
    }
    if (op & MF_STORE) a.grad[e] = scale * x;
  }
  block_partials<T>(acc, cnt, a.partials);
}

// Fixed-order reduction of the per-CTA partials (one warp).
// prepare: count (the given one, else the mask sum), 1/count, the relative normaliser (or 1), the
//   gradient scale 2 / (count * normaliser), and a zero misfit sum;
// accumulate: misfit sum += partials, loss = sum / count / normaliser.
__global__ void misfit_finalize_kernel(double* st, int n_ctas, int prepare, int relative, double count) {
  double s = 0.0, c = 0.0;
  for (int b = threadIdx.x; b < n_ctas; b += 32) {
    s += st[2 * b];
    c += st[2 * b + 1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    c += __shfl_down_sync(0xffffffffu, c, o);
  }
  if (threadIdx.x != 0) return;
  if (prepare) {
    const double n = count > 0.0 ? count : c;
    const double inv = 1.0 / fmax(n, 1e-12);
    const double den = relative ? fmax(s * inv, 1e-30) : 1.0;
    st[kStCount] = n;
    st[kStInv] = inv;
    st[kStDen] = den;
    st[kStScale] = 2.0 * inv / den;
    st[kStNum] = 0.0;
    st[kStLoss] = 0.0;
  } else {
    st[kStNum] += s;
    st[kStLoss] = st[kStNum] * st[kStInv] / st[kStDen];
  }
}

}  // namespace nw
