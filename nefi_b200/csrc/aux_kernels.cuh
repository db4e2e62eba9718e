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

// ------------------------------------------------------------------------------------------
// delta16 snapshot codec: a block of SNAP_BLOCK values x[0..31] is stored as a float anchor
// a = x[0], a float step s and 32 int16 codes. Element z decodes to
//   fmaf(s, Q[z], a),  Q[z] integer, Q[0] = 0,
// and the int16 code of element z is the second difference Q[z] - 2 Q[z-1] + Q[z-2] (Q[-1] = 0),
// so decoding is two prefix sums. The encoder takes Q[z] = rint((x[z] - a) / s) with
//   s = max( max(|x[1] - x[0]|, max_z |x[z] - 2 x[z-1] + x[z-2]|) / 32000, max_z |x[z] - a| / 2^22 ):
// the rounding error |x - decoded| is s/2 (plus one rounding of the fma), i.e. 2^-16 of the
// block's largest second difference instead of its largest value. Smooth fields (wavefields
// sampled at many cells per wavelength) have second differences several times smaller than their
// values, and the error the Laplacian of the recomputed field sees is smaller by that factor.
// Bounds: |x - a| / s <= 2^22, so |Q| and its differences are exact in float and int; each
// computed ratio (x - a) / s carries at most 0.5 of rounding error, so a code is at most
// 32000 (1 + 2^-22) + 2 (rint) + 2 (ratio rounding) < 32767 in magnitude.
//
// One thread codes one block, sequentially: the max, quantisation and differences are exact or
// single roundings of the same operands in any order, so the codes do not depend on how the work is
// split. A CTA covers D16Cta<T>::BLK consecutive blocks of one field and moves them between global
// and shared memory with coalesced 16-byte accesses; every block is a 128-byte (float) row of a
// shared tile whose 16-byte chunks are swizzled so that 8 consecutive threads reading one chunk of
// their own rows, or 8 consecutive chunks of one row, touch distinct banks.
// ------------------------------------------------------------------------------------------
template <typename T>
struct D16Cta {
  static constexpr int BLK = sizeof(T) == 8 ? 128 : 256;  // blocks per CTA (the decode's T tile: 32 KB)
  static constexpr int CH = 16 / (int)sizeof(T);           // elements of T per 16-byte chunk
};

// Element offset of chunk k (of `ch` elements) of row t in a tile of 32-element rows.
__device__ __forceinline__ int d16_chunk(int t, int k, int ch) { return t * SNAP_BLOCK + ((k ^ (t & 7)) * ch); }
// Byte offset of 16-byte chunk k (0..3) of row t in a tile of 32 int16 codes (64-byte rows).
__device__ __forceinline__ int d16_code_chunk(int t, int k) { return t * 64 + ((k ^ ((t >> 1) & 3)) << 4); }

// 16-byte loads and stores of CH elements of T through a float4 (aligned by the union).
template <typename T>
union D16Vec {
  float4 v;
  T e[16 / sizeof(T)];
};
template <typename T>
__device__ __forceinline__ void d16_ld(const T* p, T (&o)[16 / sizeof(T)]) {
  D16Vec<T> u;
  u.v = *reinterpret_cast<const float4*>(p);
#pragma unroll
  for (int i = 0; i < (int)(16 / sizeof(T)); ++i) o[i] = u.e[i];
}
template <typename T>
__device__ __forceinline__ void d16_st(T* p, const T (&o)[16 / sizeof(T)]) {
  D16Vec<T> u;
#pragma unroll
  for (int i = 0; i < (int)(16 / sizeof(T)); ++i) u.e[i] = o[i];
  *reinterpret_cast<float4*>(p) = u.v;
}

// Sets *step, *anchor and the 32 codes (packed two per word, element 2w in the low half) of the block
// x; returns false (codes 0, step and anchor NaN) if the block holds a non-finite value.
__device__ __forceinline__ bool d16_encode_block(const float (&x)[SNAP_BLOCK], unsigned (&code)[SNAP_BLOCK / 2],
                                                 float* step, float* anchor) {
  bool finite = true;
#pragma unroll
  for (int z = 0; z < SNAP_BLOCK; ++z) finite = finite && fabsf(x[z]) <= 3.0e38f;
  if (!finite) {
#pragma unroll
    for (int w = 0; w < SNAP_BLOCK / 2; ++w) code[w] = 0u;
    *step = *anchor = __int_as_float(0x7fc00000);
    return false;
  }
  const float a = x[0];
  float m = 0.f, r = 0.f, dxm1 = 0.f;  // max |second difference|, max |x - a|, x[z-1] - x[z-2]
#pragma unroll
  for (int z = 1; z < SNAP_BLOCK; ++z) {
    const float dx = x[z] - x[z - 1];
    const float d2 = z >= 2 ? dx - dxm1 : dx;
    m = fmaxf(m, fabsf(d2));
    r = fmaxf(r, fabsf(x[z] - a));
    dxm1 = dx;
  }
  const float s = fmaxf(fmaxf(m * (1.f / 32000.f), r * 0x1p-22f), 1.17549435e-38f);
  const float inv = 1.f / s;
  int qm1 = 0, qm2 = 0;  // Q[z-1], Q[z-2]
#pragma unroll
  for (int z = 0; z < SNAP_BLOCK; ++z) {
    const int q = z == 0 ? 0 : (int)rintf((x[z] - a) * inv);
    int d = z >= 2 ? q - 2 * qm1 + qm2 : (z == 1 ? q : 0);
    d = max(-32767, min(32767, d));
    const unsigned h = (unsigned)(unsigned short)(short)d;
    if (z & 1) code[z >> 1] |= h << 16;
    else code[z >> 1] = h;
    qm2 = qm1;
    qm1 = q;
  }
  *step = s;
  *anchor = a;
  return true;
}

// The 32 values of a block from its codes, step and anchor (two running sums, exact in int).
__device__ __forceinline__ void d16_decode_block(const unsigned (&code)[SNAP_BLOCK / 2], float s, float a,
                                                 float (&v)[SNAP_BLOCK]) {
  int d1 = 0, q = 0;
#pragma unroll
  for (int z = 0; z < SNAP_BLOCK; ++z) {
    const int c = (int)(short)(unsigned short)(z & 1 ? code[z >> 1] >> 16 : code[z >> 1] & 0xffffu);
    d1 += c;
    q += d1;
    v[z] = fmaf(s, (float)q, a);
  }
}

// Encodes snapshot slots with one launch: grid.z = slot (0: l0 = p^{n0}; 1: l0 - lm1; 2, 3: the
// PML face fields f0, f1), grid.y = shot, grid.x = groups of D16Cta<T>::BLK blocks. Slot k of shot f
// occupies blocks (k * n_shots + f) * nblk of vals / steps / anchors. Every field holds nblk whole
// blocks (its length is a multiple of SNAP_BLOCK).
template <typename T>
__global__ void __launch_bounds__(256) snap_encode_d16(const T* __restrict__ lm1, const T* __restrict__ l0,
                                                       const T* __restrict__ f0, const T* __restrict__ f1,
                                                       long long field, int nblk, short* __restrict__ vals,
                                                       float* __restrict__ steps, float* __restrict__ anchors) {
  constexpr int BLK = D16Cta<T>::BLK, CH = D16Cta<T>::CH;
  __shared__ __align__(16) float tile[BLK * SNAP_BLOCK];  // the values as float; reused for the codes
  const int f = blockIdx.y, slot = blockIdx.z, n_shots = gridDim.y;
  const long long bb = (long long)blockIdx.x * BLK;  // first block of this CTA within the field
  const int nb = (int)min((long long)BLK, (long long)nblk - bb);
  const T* src = slot == 0 ? l0 : (slot == 1 ? l0 : (slot == 2 ? f0 : f1));
  const T* sub = slot == 1 ? lm1 : nullptr;
  const long long e0 = (long long)f * field + bb * SNAP_BLOCK;  // first element
  // staging: 16-byte chunks of T in field order, converted to float, into the swizzled tile
  constexpr int CPR = SNAP_BLOCK / CH;
  const int n_chunks = nb * CPR;
#pragma unroll 4
  for (int c = threadIdx.x; c < n_chunks; c += 256) {
    const int row = c / CPR, k = c - row * CPR;
    T v[CH];
    d16_ld<T>(src + e0 + (long long)c * CH, v);
    if (sub) {
      T w[CH];
      d16_ld<T>(sub + e0 + (long long)c * CH, w);
#pragma unroll
      for (int i = 0; i < CH; ++i) v[i] = v[i] - w[i];
    }
    // the chunk's CH floats sit inside one 16-byte float chunk of the row
    const int z = k * CH;
    float* dst = tile + d16_chunk(row, z >> 2, 4) + (z & 3);
#pragma unroll
    for (int i = 0; i < CH; ++i) dst[i] = (float)v[i];
  }
  __syncthreads();
  const int t = threadIdx.x;
  unsigned code[SNAP_BLOCK / 2];
  if (t < nb) {
    float x[SNAP_BLOCK];
#pragma unroll
    for (int k = 0; k < SNAP_BLOCK / 4; ++k) {
      const float4 q = *reinterpret_cast<const float4*>(tile + d16_chunk(t, k, 4));
      x[4 * k] = q.x; x[4 * k + 1] = q.y; x[4 * k + 2] = q.z; x[4 * k + 3] = q.w;
    }
    float s, a;
    if (!d16_encode_block(x, code, &s, &a)) atomicExch(&g_status, 4);
    const long long blk = ((long long)slot * n_shots + f) * nblk + bb + t;
    steps[blk] = s;
    anchors[blk] = a;
  }
  __syncthreads();  // every row has been read: the tile takes the codes (64-byte rows)
  unsigned char* ct = reinterpret_cast<unsigned char*>(tile);
  if (t < nb) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      *reinterpret_cast<uint4*>(ct + d16_code_chunk(t, k)) =
          make_uint4(code[4 * k], code[4 * k + 1], code[4 * k + 2], code[4 * k + 3]);
  }
  __syncthreads();
  uint4* out = reinterpret_cast<uint4*>(vals + ((((long long)slot * n_shots + f) * nblk + bb) * SNAP_BLOCK));
  for (int c = threadIdx.x; c < nb * 4; c += 256)
    out[c] = *reinterpret_cast<const uint4*>(ct + d16_code_chunk(c >> 2, c & 3));
}

// Number of leading elements of block b (elements 32 b .. 32 b + 31 of a field in the ghost layout)
// that are cells of the padded grid grown by `ex` cells at the high end of axis 0 and `ez` at the high
// end of the contiguous axis (a face field of the PML: face P of an axis sits in the first ghost row
// or column). Rows start on multiples of SNAP_BLOCK elements (the guard and the row pitch are), so a
// block lies in one row and its grid cells are a prefix of it.
template <typename T>
__device__ __forceinline__ int d16_grid_prefix(const KGrid<T>& g, int ndim, long long b, int ex, int ez) {
  long long u = b * SNAP_BLOCK - g.origin;
  if (u < 0) return 0;
  const long long x = u / g.s0;
  u -= x * g.s0;
  if (x >= g.n0 + ex) return 0;
  long long n_inner = g.n1 + ez;
  if (ndim == 3) {
    const long long y = u / g.s1;
    if (y >= g.n1) return 0;
    u -= y * g.s1;
    n_inner = g.n2 + ez;
  }
  return (int)max(0LL, min((long long)SNAP_BLOCK, n_inner - u));
}

// Writes a CTA's tile of decoded rows (T, swizzled 16-byte chunks) to out, in coalesced chunks, only
// the first len[row] elements of each row.
template <typename T>
__device__ __forceinline__ void d16_store_rows(const T* tile, const int* len, int nb, T* __restrict__ out) {
  constexpr int CH = D16Cta<T>::CH, CPR = SNAP_BLOCK / CH;
  for (int c = threadIdx.x; c < nb * CPR; c += 256) {
    const int row = c / CPR, k = c - row * CPR;
    const int n = len[row] - k * CH;  // valid elements of this chunk
    if (n <= 0) continue;
    const T* src = tile + d16_chunk(row, k, CH);
    T* dst = out + (long long)row * SNAP_BLOCK + k * CH;
    if (n >= CH) {
      T v[CH];
      d16_ld<T>(src, v);
      d16_st<T>(dst, v);
    } else {
      for (int i = 0; i < n; ++i) dst[i] = src[i];
    }
  }
}

// Decodes with one launch: grid.z = 0 decodes slots 0 and 1 of each block together (l0_out = p^{n0},
// lm1_out = p^{n0} - difference, in T like the separate-slot codecs), grid.z = 1 (PML) the face
// slots 2 and 3 into f0_out, f1_out; grid.y = shot, grid.x = groups of D16Cta<T>::BLK blocks. Only the
// elements that hold grid cells (faces) are written: a code relative to the block's anchor returns
// a zero outside the grid only to within half a step, and the cells outside the grid must stay exact
// zeros (the Laplacian's zero padding).
template <typename T>
__global__ void __launch_bounds__(256) snap_decode_d16(const short* __restrict__ vals, const float* __restrict__ steps,
                                                       const float* __restrict__ anchors, int nblk, long long field,
                                                       KGrid<T> g, int ndim,
                                                       T* __restrict__ lm1_out, T* __restrict__ l0_out,
                                                       T* __restrict__ f0_out, T* __restrict__ f1_out) {
  constexpr int BLK = D16Cta<T>::BLK, CH = D16Cta<T>::CH;
  // the two slots' codes (64-byte rows), then the decoded rows of one output (T)
  __shared__ __align__(16) unsigned char smem[BLK * SNAP_BLOCK * sizeof(T)];
  __shared__ int len0[BLK], len1[BLK];
  static_assert(2 * BLK * 64 <= BLK * SNAP_BLOCK * (int)sizeof(T), "code tiles fit the row tile");
  const int f = blockIdx.y, pair = blockIdx.z, n_shots = gridDim.y;
  const long long bb = (long long)blockIdx.x * BLK;
  const int nb = (int)min((long long)BLK, (long long)nblk - bb);
  const long long blkA = ((long long)(2 * pair) * n_shots + f) * nblk + bb;
  const long long blkB = ((long long)(2 * pair + 1) * n_shots + f) * nblk + bb;
  unsigned char* ca = smem;
  unsigned char* cb = smem + BLK * 64;
  {
    const uint4* ga = reinterpret_cast<const uint4*>(vals + blkA * SNAP_BLOCK);
    const uint4* gb = reinterpret_cast<const uint4*>(vals + blkB * SNAP_BLOCK);
#pragma unroll 4
    for (int c = threadIdx.x; c < nb * 4; c += 256) {
      const uint4 qa = ga[c], qb = gb[c];
      *reinterpret_cast<uint4*>(ca + d16_code_chunk(c >> 2, c & 3)) = qa;
      *reinterpret_cast<uint4*>(cb + d16_code_chunk(c >> 2, c & 3)) = qb;
    }
  }
  const int t = threadIdx.x;
  float sa = 1.f, aa = 0.f, sb = 1.f, ab = 0.f;
  if (t < nb) {
    sa = steps[blkA + t];
    aa = anchors[blkA + t];
    sb = steps[blkB + t];
    ab = anchors[blkB + t];
    if (!(sa > 0.f && sa <= 3.0e38f && sb > 0.f && sb <= 3.0e38f && fabsf(aa) <= 3.0e38f && fabsf(ab) <= 3.0e38f))
      atomicExch(&g_status, 4);
    const long long b = bb + t;
    if (pair == 0) {
      len0[t] = d16_grid_prefix(g, ndim, b, 0, 0);
    } else {
      len0[t] = d16_grid_prefix(g, ndim, b, 1, 0);
      len1[t] = d16_grid_prefix(g, ndim, b, 0, 1);
    }
  }
  __syncthreads();
  unsigned qa[SNAP_BLOCK / 2], qb[SNAP_BLOCK / 2];
  if (t < nb) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint4 u = *reinterpret_cast<const uint4*>(ca + d16_code_chunk(t, k));
      const uint4 w = *reinterpret_cast<const uint4*>(cb + d16_code_chunk(t, k));
      qa[4 * k] = u.x; qa[4 * k + 1] = u.y; qa[4 * k + 2] = u.z; qa[4 * k + 3] = u.w;
      qb[4 * k] = w.x; qb[4 * k + 1] = w.y; qb[4 * k + 2] = w.z; qb[4 * k + 3] = w.w;
    }
  }
  __syncthreads();  // the code tiles are read: the smem takes the decoded rows
  T* tile = reinterpret_cast<T*>(smem);
  const long long e0 = (long long)f * field + bb * SNAP_BLOCK;
  float va[SNAP_BLOCK];
  if (t < nb) {
    d16_decode_block(qa, sa, aa, va);
#pragma unroll
    for (int k = 0; k < SNAP_BLOCK / CH; ++k) {
      T o[CH];
#pragma unroll
      for (int i = 0; i < CH; ++i) o[i] = (T)va[k * CH + i];
      d16_st<T>(tile + d16_chunk(t, k, CH), o);
    }
  }
  __syncthreads();
  d16_store_rows<T>(tile, len0, nb, (pair == 0 ? l0_out : f0_out) + e0);
  __syncthreads();
  if (t < nb) {
    float vb[SNAP_BLOCK];
    d16_decode_block(qb, sb, ab, vb);
#pragma unroll
    for (int k = 0; k < SNAP_BLOCK / CH; ++k) {
      T o[CH];
#pragma unroll
      for (int i = 0; i < CH; ++i) {
        const int z = k * CH + i;
        o[i] = pair == 0 ? (T)va[z] - (T)vb[z] : (T)vb[z];
      }
      d16_st<T>(tile + d16_chunk(t, k, CH), o);
    }
  }
  __syncthreads();
  d16_store_rows<T>(tile, pair == 0 ? len0 : len1, nb, (pair == 0 ? lm1_out : f1_out) + e0);
}

}  // namespace nw
