// aux_kernels.cuh — preparation, reduction and snapshot kernels of the leapfrog propagator.
#pragma once
#include "kernels.cuh"

namespace nw {

// Physical-grid index helpers: a padded cell (x, y, z) maps to the physical cell
// clamp(x - a, 0, n - 1) per axis under replicate padding (nefi/physics/wave.py:231-240).
struct PadMap {
  int a0, a1, a2;  // layer widths
  int m0, m1, m2;  // physical extents (m2 = 1 in 2-D)
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// c2dt2[cell] = c[pad_replicate(cell)]^2 * dt2 over all padded cells (2-D: n2 = 1).
template <typename T>
__global__ void medium_kernel(KGrid<T> g, PadMap pm, const T* __restrict__ c, T dt2, int ndim,
                              T* __restrict__ out) {
  const long long cells = (long long)g.n0 * g.n1 * g.n2;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < cells;
       t += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(t % g.n2);
    const int y = (int)((t / g.n2) % g.n1);
    const int x = (int)(t / ((long long)g.n2 * g.n1));
    long long src, dst;
    if (ndim == 2) {  // (x, y) are the two axes, z == 0
      const int i = clampi(x - pm.a0, 0, pm.m0 - 1), j = clampi(y - pm.a1, 0, pm.m1 - 1);
      src = (long long)i * pm.m1 + j;
      dst = g.origin + (long long)x * g.s0 + y;
    } else {
      const int i = clampi(x - pm.a0, 0, pm.m0 - 1), j = clampi(y - pm.a1, 0, pm.m1 - 1),
                k = clampi(z - pm.a2, 0, pm.m2 - 1);
      src = ((long long)i * pm.m1 + j) * pm.m2 + k;
      dst = g.origin + (long long)x * g.s0 + (long long)y * g.s1 + z;
    }
    const T cv = c[src];
    const T c2 = cv * cv;
    out[dst] = c2 * dt2;
  }
}

// Zero-padded copy of per-shot physical fields into ghost-layout levels.
template <typename T>
__global__ void pad_zero_kernel(KGrid<T> g, PadMap pm, int ndim, const T* __restrict__ p0,
                                T* __restrict__ lvl) {
  const int s = blockIdx.y;
  const long long cells = (long long)pm.m0 * pm.m1 * pm.m2;
  const T* src = p0 + (long long)s * cells;
  T* dst = lvl + (long long)s * g.field;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < cells;
       t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % pm.m2);
    const int j = (int)((t / pm.m2) % pm.m1);
    const int i = (int)(t / ((long long)pm.m2 * pm.m1));
    long long d;
    if (ndim == 2) d = g.origin + (long long)(i + pm.a0) * g.s0 + (j + pm.a1);
    else d = g.origin + (long long)(i + pm.a0) * g.s0 + (long long)(j + pm.a1) * g.s1 + (k + pm.a2);
    dst[d] = src[t];
  }
}

template <typename T, int R>
__device__ __forceinline__ T lap_at(const KGrid<T>& g, const T* __restrict__ p, long long i, int ndim) {
  T l;
  if (ndim == 2) {
    l = g.wc * p[i] + g.w1a * (p[i - g.s0] + p[i + g.s0]) + g.w1b * (p[i - 1] + p[i + 1]);
    if (R == 2) l += g.w2a * (p[i - 2 * g.s0] + p[i + 2 * g.s0]) + g.w2b * (p[i - 2] + p[i + 2]);
  } else {
    l = g.wc * p[i] + g.w1a * (p[i - g.s0] + p[i + g.s0]) + g.w1b * (p[i - g.s1] + p[i + g.s1]) +
        g.w1c * (p[i - 1] + p[i + 1]);
    if (R == 2)
      l += g.w2a * (p[i - 2 * g.s0] + p[i + 2 * g.s0]) + g.w2b * (p[i - 2 * g.s1] + p[i + 2 * g.s1]) +
           g.w2c * (p[i - 2] + p[i + 2]);
  }
  return l;
}

__device__ __forceinline__ bool cell_of(long long t, int n0, int n1, int n2, int ndim, int& x, int& y,
                                        int& z) {
  z = (int)(t % n2);
  y = (int)((t / n2) % n1);
  x = (int)(t / ((long long)n2 * n1));
  return true;
}

template <typename T>
__device__ __forceinline__ long long ghost_index(const KGrid<T>& g, int ndim, int x, int y, int z) {
  return ndim == 2 ? g.origin + (long long)x * g.s0 + y
                   : g.origin + (long long)x * g.s0 + (long long)y * g.s1 + z;
}

// p^-1 = p^0 + (0.5 c2dt2) * Lap p^0 over all padded cells (nefi/physics/wave.py:850).
template <typename T, int R>
__global__ void initial_prev_kernel(KGrid<T> g, int ndim, const T* __restrict__ C,
                                    const T* __restrict__ p0, T* __restrict__ pm1) {
  const int s = blockIdx.y;
  const long long cells = (long long)g.n0 * g.n1 * g.n2;
  const T* p = p0 + (long long)s * g.field;
  T* out = pm1 + (long long)s * g.field;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < cells;
       t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    cell_of(t, g.n0, g.n1, g.n2, ndim, x, y, z);
    const long long i = ghost_index(g, ndim, x, y, z);
    const T h = T(0.5) * C[i];
    out[i] = p[i] + h * lap_at<T, R>(g, p, i, ndim);
  }
}

// Dirichlet condition of time reversal: lvl[cells[c]] = w0 traces[c, j0] + w1 traces[c, j1] (the
// traces at a reversed time, linear between samples; products and sum rounded separately, as the
// reference's scalar-times-tensor expression is).
template <typename T>
__global__ void dirichlet_kernel(T* __restrict__ lvl, const int64_t* __restrict__ cells, int n_cells,
                                 const T* __restrict__ traces, int n_t, int j0, int j1, T w0, T w1) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  const T* tr = traces + (long long)c * n_t;
  lvl[cells[c]] = add_rn(mul_rn(w0, tr[j0]), mul_rn(w1, tr[j1]));
}

// mu = q / C on the padded grid of shot blockIdx.y (q = C mu is the variable the adjoint steps
// advance). Ghost cells are left untouched (the caller zeroes them).
template <typename T>
__global__ void unscale_kernel(KGrid<T> g, int ndim, const T* __restrict__ C, const T* __restrict__ q,
                               T* __restrict__ out) {
  const long long so = (long long)blockIdx.y * g.field;
  const long long cells = (long long)g.n0 * g.n1 * g.n2;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < cells;
       t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    cell_of(t, g.n0, g.n1, g.n2, ndim, x, y, z);
    const long long i = ghost_index(g, ndim, x, y, z);
    out[so + i] = q[so + i] / C[i];
  }
}

// Adjoint of the initial state: lambda^-1 = -B0 mu^1,
// grad_p0p = lambda^0 + lambda^-1 + Lap(0.5 C lambda^-1), cropped to the physical grid;
// optionally acc[s / spa] += C * 0.5 lambda^-1 Lap p^0 (the accumulators hold C dJ/dC, as the
// adjoint steps leave them). blockIdx.y is an accumulator group whose
// shots a thread visits in order, so no two threads add into the same accumulator cell.
template <typename T, int R>
__global__ void initial_adjoint_kernel(KGrid<T> g, PadMap pm, int ndim, const T* __restrict__ C,
                                       const T* __restrict__ B, int b_one, int n_shots, int spa,
                                       const T* __restrict__ lam0, const T* __restrict__ mu1,
                                       const T* __restrict__ p0, T* __restrict__ grad_p0,
                                       T* __restrict__ acc) {
  const int grp = blockIdx.y;
  const long long cells = (long long)g.n0 * g.n1 * g.n2;
  const long long pcells = (long long)pm.m0 * pm.m1 * pm.m2;
  T* ga = acc ? acc + (long long)grp * g.field : nullptr;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < cells;
       t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    cell_of(t, g.n0, g.n1, g.n2, ndim, x, y, z);
    const long long i = ghost_index(g, ndim, x, y, z);
    int pi, pj, pk;
    if (ndim == 2) { pi = x - pm.a0; pj = y - pm.a1; pk = 0; }
    else { pi = x - pm.a0; pj = y - pm.a1; pk = z - pm.a2; }
    const bool phys = !(pi < 0 || pi >= pm.m0 || pj < 0 || pj >= pm.m1 || pk < 0 || pk >= pm.m2);
    for (int s = grp * spa; s < min(n_shots, (grp + 1) * spa); ++s) {
      const long long so = (long long)s * g.field;
      const T* m = mu1 + so;
      auto lm1 = [&](long long k) -> T {
        const T b = (b_one || B == nullptr) ? T(1) : B[k];
        return -(b * m[k]);
      };
      auto hl = [&](long long k) -> T { return (T(0.5) * C[k]) * lm1(k); };
      const T l = lm1(i);
      if (ga) ga[i] += C[i] * ((T(0.5) * l) * lap_at<T, R>(g, p0 + so, i, ndim));
      if (!phys) continue;
      T lh;
      if (ndim == 2) {
        lh = g.wc * hl(i) + g.w1a * (hl(i - g.s0) + hl(i + g.s0)) + g.w1b * (hl(i - 1) + hl(i + 1));
        if (R == 2) lh += g.w2a * (hl(i - 2 * g.s0) + hl(i + 2 * g.s0)) + g.w2b * (hl(i - 2) + hl(i + 2));
      } else {
        lh = g.wc * hl(i) + g.w1a * (hl(i - g.s0) + hl(i + g.s0)) + g.w1b * (hl(i - g.s1) + hl(i + g.s1)) +
             g.w1c * (hl(i - 1) + hl(i + 1));
        if (R == 2)
          lh += g.w2a * (hl(i - 2 * g.s0) + hl(i + 2 * g.s0)) + g.w2b * (hl(i - 2 * g.s1) + hl(i + 2 * g.s1)) +
                g.w2c * (hl(i - 2) + hl(i + 2));
      }
      const long long pidx = ((long long)pi * pm.m1 + pj) * pm.m2 + pk;
      grad_p0[(long long)s * pcells + pidx] = (lam0[so + i] + l) + lh;
    }
  }
}

// grad_c[phys] (+)= 2 c dt2 * dJ/dC, dJ/dC = sum_acc sum_{padded cells -> phys} g_acc[cell] / C, in
// float64. A warp takes 32 consecutive physical cells: each lane sums its cell when a single
// padded cell maps to it (the interior); cells on the border of the physical grid, onto which a
// whole strip or block of the absorbing layer folds (up to (a+1)^ndim padded cells), are then
// summed by the whole warp, lanes striding the block in a fixed order and combining by a fixed
// shuffle tree, so the result is reproducible and no thread walks a corner block alone.
template <typename T>
__global__ void reduce_grad_kernel(KGrid<T> g, PadMap pm, int ndim, const T* __restrict__ c,
                                   double dt2, int n_acc, const T* __restrict__ gs,
                                   int accumulate, double* __restrict__ out) {
  const long long pcells = (long long)pm.m0 * pm.m1 * pm.m2;
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long n_warps = ((long long)gridDim.x * blockDim.x) >> 5;
  // padded range mapping onto physical index i along an axis of width m with layer a
  auto lo = [](int i, int a, int m) { return i == 0 ? 0 : i + a; };
  auto hi = [](int i, int a, int m) { return i == m - 1 ? m + 2 * a - 1 : i + a; };
  auto finish = [&](long long t, double acc) {
    // acc = C dJ/dC summed over the padded cells that replicate c[t], all with C = c^2 dt^2
    const double cd = (double)c[t];
    const double v = 2.0 * cd * dt2 * (acc / (cd * cd * dt2));
    out[t] = accumulate ? out[t] + v : v;
  };
  for (long long base = warp * 32; base < pcells; base += n_warps * 32) {
    const long long t = base + lane;
    int x0 = 0, x1 = -1, y0 = 0, y1 = 0, z0 = 0, z1 = 0;
    if (t < pcells) {
      const int k = (int)(t % pm.m2);
      const int j = (int)((t / pm.m2) % pm.m1);
      const int i = (int)(t / ((long long)pm.m2 * pm.m1));
      x0 = lo(i, pm.a0, pm.m0); x1 = hi(i, pm.a0, pm.m0);
      y0 = lo(j, pm.a1, pm.m1); y1 = hi(j, pm.a1, pm.m1);
      z0 = ndim == 3 ? lo(k, pm.a2, pm.m2) : 0; z1 = ndim == 3 ? hi(k, pm.a2, pm.m2) : 0;
    }
    const bool single = t < pcells && x0 == x1 && y0 == y1 && z0 == z1;
    if (single) {
      const long long idx = ghost_index(g, ndim, x0, y0, z0);
      double acc = 0.0;
      for (int s = 0; s < n_acc; ++s) acc += (double)gs[(long long)s * g.field + idx];
      finish(t, acc);
    }
    unsigned todo = __ballot_sync(0xffffffffu, t < pcells && !single);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const int bx0 = __shfl_sync(0xffffffffu, x0, src), bx1 = __shfl_sync(0xffffffffu, x1, src);
      const int by0 = __shfl_sync(0xffffffffu, y0, src), by1 = __shfl_sync(0xffffffffu, y1, src);
      const int bz0 = __shfl_sync(0xffffffffu, z0, src), bz1 = __shfl_sync(0xffffffffu, z1, src);
      const int ny = by1 - by0 + 1, nz = bz1 - bz0 + 1;
      const long long nb = (long long)(bx1 - bx0 + 1) * ny * nz;
      double part = 0.0;
      for (long long q = lane; q < nb; q += 32) {
        const int z = bz0 + (int)(q % nz), y = by0 + (int)((q / nz) % ny), x = bx0 + (int)(q / ((long long)nz * ny));
        const long long idx = ghost_index(g, ndim, x, y, z);
        for (int s = 0; s < n_acc; ++s) part += (double)gs[(long long)s * g.field + idx];
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
      if (lane == src) finish(t, part);
    }
  }
}

// Zero the ghost cells of n_fields consecutive fields (a warp per storage row): whole rows
// outside the grid and the tail [n_last, ld) of every data row. Interior cells are untouched.
template <typename T>
__global__ void zero_ghosts_kernel(T* __restrict__ base, long long field, int guard, long long n_rows,
                                   int ld, int n_last, int ndim, int r, int n0, int n1,
                                   int rows_per_plane, long long n_fields) {
  const long long warps = (long long)gridDim.x * (blockDim.x / 32);
  const int lane = threadIdx.x & 31;
  for (long long w = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; w < n_rows * n_fields;
       w += warps) {
    const long long f = w / n_rows, row = w % n_rows;
    bool ghost_row;
    if (ndim == 2) {
      ghost_row = row < r || row >= r + n0;
    } else {
      const long long plane = row / rows_per_plane, y = row % rows_per_plane;
      ghost_row = plane < r || plane >= r + n0 || y >= n1;
    }
    if (row == 0)
      for (int z = lane; z < guard; z += 32) base[f * field + z] = T(0);
    T* p = base + f * field + guard + row * ld;
    for (int z = ghost_row ? lane : n_last + lane; z < ld; z += 32) p[z] = T(0);
  }
}

// ------------------------------------------------------------------------------------------
// Snapshot codec: blocks of SNAP_BLOCK = 32 contiguous elements of one field (one warp), each
// stored as 16-bit values with one float scale per block:
//   fp16 / bf16: power-of-two scale (exact to apply), 11- / 8-bit mantissas;
//   fixed16:     int16 mantissas with scale = block max / 32767 (block floating point), whose
//                absolute error is 2^-16 of the block maximum.
// ------------------------------------------------------------------------------------------
constexpr int SNAP_BLOCK = 32;
constexpr int CODEC_F16 = 1, CODEC_BF16 = 2, CODEC_I16 = 3;

template <int K>
struct Codec;
template <>
struct Codec<CODEC_F16> {
  using H = __half;
  static __device__ __forceinline__ float scale(float mx) {
    int e;
    frexpf(mx, &e);  // mx <= 2^e; |v / scale| <= 2^15 < 65504
    return ldexpf(1.f, max(-126, min(127, e - 15)));
  }
  static __device__ __forceinline__ H enc(float v, float inv) { return __float2half_rn(v * inv); }
  static __device__ __forceinline__ float dec(H q, float s) { return __half2float(q) * s; }
};
template <>
struct Codec<CODEC_BF16> {
  using H = __nv_bfloat16;
  static __device__ __forceinline__ float scale(float mx) {
    int e;
    frexpf(mx, &e);
    return ldexpf(1.f, max(-126, min(127, e)));
  }
  static __device__ __forceinline__ H enc(float v, float inv) { return __float2bfloat16_rn(v * inv); }
  static __device__ __forceinline__ float dec(H q, float s) { return __bfloat162float(q) * s; }
};
template <>
struct Codec<CODEC_I16> {
  using H = short;
  static __device__ __forceinline__ float scale(float mx) { return fmaxf(mx / 32767.f, 1.17549435e-38f); }
  static __device__ __forceinline__ H enc(float v, float inv) {
    return (short)fminf(32767.f, fmaxf(-32767.f, rintf(v * inv)));
  }
  static __device__ __forceinline__ float dec(H q, float s) { return (float)q * s; }
};

__device__ int g_status;  // sticky device status word (NW_ERR_* or 0)

// Encodes src (or src - sub when sub != nullptr: the level difference, whose small magnitude
// would be lost if both levels were rounded to 16 bits separately). One warp per SNAP_WARP_BLOCKS
// consecutive blocks, their loads issued together; grid.x covers the blocks of one field, grid.y the
// fields. Each block is coded exactly as on its own.
constexpr int SNAP_WARP_BLOCKS = 4;
template <typename T, int K>
__global__ void __launch_bounds__(256) snap_encode(const T* __restrict__ src, const T* __restrict__ sub,
                                                   long long field, int nblk,
                                                   typename Codec<K>::H* __restrict__ vals,
                                                   float* __restrict__ scales) {
  const int f = blockIdx.y;
  const long long b0 = ((long long)blockIdx.x * 8 + (threadIdx.x >> 5)) * SNAP_WARP_BLOCKS;
  if (b0 >= nblk) return;
  const int lane = threadIdx.x & 31;
  float v[SNAP_WARP_BLOCKS];
#pragma unroll
  for (int u = 0; u < SNAP_WARP_BLOCKS; ++u) {
    const long long e = (b0 + u) * SNAP_BLOCK + lane;
    v[u] = 0.f;
    if (b0 + u < nblk && e < field) {
      const long long i = (long long)f * field + e;
      v[u] = (float)(sub ? src[i] - sub[i] : src[i]);
    }
  }
#pragma unroll
  for (int u = 0; u < SNAP_WARP_BLOCKS; ++u) {
    const long long b = b0 + u;
    if (b >= nblk) break;  // warp-uniform
    const bool bad = !(fabsf(v[u]) <= 3.0e38f);  // NaN or Inf
    float mx = fabsf(v[u]);
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const bool any_bad = __any_sync(0xffffffffu, bad);
    float s = 1.f;
    if (any_bad) {
      s = __int_as_float(0x7fc00000);
      if (lane == 0) atomicExch(&g_status, 4);
    } else if (mx > 0.f) {
      s = Codec<K>::scale(mx);
    }
    const float inv = any_bad ? 0.f : 1.f / s;
    vals[(long long)f * nblk * SNAP_BLOCK + b * SNAP_BLOCK + lane] = Codec<K>::enc(v[u], inv);
    if (lane == 0) scales[(long long)f * nblk + b] = s;
  }
}

// Decodes into dst (or dst = minuend - decoded when minuend != nullptr, undoing the difference
// encoding of snap_encode); SNAP_WARP_BLOCKS blocks per warp like the encoder.
template <typename T, int K>
__global__ void __launch_bounds__(256) snap_decode(const typename Codec<K>::H* __restrict__ vals,
                                                   const float* __restrict__ scales, int nblk,
                                                   long long field, const T* __restrict__ minuend,
                                                   T* __restrict__ dst) {
  const int f = blockIdx.y;
  const long long b0 = ((long long)blockIdx.x * 8 + (threadIdx.x >> 5)) * SNAP_WARP_BLOCKS;
  if (b0 >= nblk) return;
  const int lane = threadIdx.x & 31;
  float sc[SNAP_WARP_BLOCKS];
  typename Codec<K>::H q[SNAP_WARP_BLOCKS];
  T mn[SNAP_WARP_BLOCKS];
#pragma unroll
  for (int u = 0; u < SNAP_WARP_BLOCKS; ++u) {
    const long long b = b0 + u;
    const long long e = b * SNAP_BLOCK + lane;
    sc[u] = 1.f;
    mn[u] = T(0);
    if (b < nblk) {
      sc[u] = scales[(long long)f * nblk + b];
      q[u] = vals[(long long)f * nblk * SNAP_BLOCK + b * SNAP_BLOCK + lane];
      if (minuend && e < field) mn[u] = minuend[(long long)f * field + e];
    }
  }
#pragma unroll
  for (int u = 0; u < SNAP_WARP_BLOCKS; ++u) {
    const long long b = b0 + u;
    if (b >= nblk) break;
    if (!(sc[u] > 0.f && sc[u] <= 3.0e38f) && lane == 0) atomicExch(&g_status, 4);
    const long long e = b * SNAP_BLOCK + lane;
    if (e >= field) continue;
    const T v = (T)Codec<K>::dec(q[u], sc[u]);
    dst[(long long)f * field + e] = minuend ? mn[u] - v : v;
  }
}

}  // namespace nw
