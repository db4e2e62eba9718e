// kernels.cuh — device code of the acoustic leapfrog propagator (sm_100a).
//
// Scheme (nefi/physics/wave.py:529-552), per cell and shot:
//   p^{n+1} = A * ( 2 p^n - B p^{n-1} + C * Lap(p^n) + S w(n) ),   C = c^2 dt^2,
// with A = B = 1 outside the absorbing layer. Its exact discrete adjoint, with mu^n = A lambda^n:
//   mu^n = A * ( R^T g_n + 2 mu^{n+1} + Lap(C mu^{n+1}) - B mu^{n+2} ),
//   dJ/dC += mu^{n+1} * Lap(p^n), with Lap(p^n) stored by the forward step that computed it.
// The kernels advance q = C mu instead, which obeys the forward's own recursion
//   q^n = A * ( 2 q^{n+1} - B q^{n+2} + C * Lap(q^{n+1}) + C R^T g_n ),
// so one stencil serves both directions, and accumulate C dJ/dC = sum_n q^{n+1} Lap(p^n).
// Fields live in the ghost layout (see nw_grid in include/nefi_wave.h): every neighbour read is
// in bounds and reads zero outside the padded grid, so the stencils carry no boundary branches.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace nw {

// Arithmetic with a fixed rounding sequence: the compiler may not fuse or reorder these, so a
// stencil written with them gives bitwise the same result in every kernel instantiation (tile
// shape, vector width) that evaluates it.
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// Kernel-side copy of the grid geometry, passed by value.
template <typename T>
struct KGrid {
  int n0, n1, n2;           // padded extents (2-D: n2 = 1, axis 1 contiguous)
  int lo0, lo1, lo2;        // interior box [lo, hi) outside the absorbing layer
  int hi0, hi1, hi2;
  long long s0, s1;         // element strides of axis 0 and axis 1 (3-D); contiguous axis = 1
  long long origin;         // offset of cell (0,..,0)
  long long field;          // elements per field (shot stride inside a level)
  T wc, w1a, w1b, w1c;      // Laplacian weights: centre, +-1 per axis
  T w2a, w2b, w2c;          // +-2 per axis (order 4)
};

// Everything one 3-D step reads and writes: forward (p) or adjoint (q = C mu), as in step2d.
template <typename T>
struct Step3 {
  const T* __restrict__ prev;   // forward p^{n-1} | adjoint q^{n+2} (shot 0; shots follow at +field)
  const T* __restrict__ cur;    // forward p^n     | adjoint q^{n+1}
  T* __restrict__ next;         // forward p^{n+1} | adjoint q^n
  const T* __restrict__ C;      // c^2 dt^2
  const T* __restrict__ A;      // absorbing coefficients or nullptr
  const T* __restrict__ B;
  int b_one;                    // forward: use B = 1 on the previous level (first Cerjan step)
  int apply_a;                  // adjoint: A applies (n >= 1)
  // forward source: one multilinear stencil per shot
  const int* __restrict__ src_corner;  // (shots, ndim) or nullptr
  const T* __restrict__ src_w;         // (shots, 2^ndim)
  const T* __restrict__ wavelet;       // (n_steps,)
  int n;                               // step index
  // forward receivers sampled from level n when `traces` != nullptr
  T* __restrict__ traces;              // (shots, n_rec, n_t)
  const int64_t* __restrict__ rec_idx;
  const T* __restrict__ rec_w;
  int n_rec, n_t, j;
  T* __restrict__ lap_out;             // forward, non-null: also store Lap p^n (the gradient factor)
  const T* __restrict__ lap;           // adjoint: Lap p^n as the forward stored it (nullptr: no gradient)
  T* __restrict__ grad;                // adjoint: per-shot accumulators of C dJ/dC
};

__device__ __forceinline__ long long global_thread_in_shot() {
  return ((long long)blockIdx.y * gridDim.x + blockIdx.x) * (blockDim.x * blockDim.y) +
         threadIdx.y * blockDim.x + threadIdx.x;
}

// Receiver gather of one level for shot s: traces[s, r, j] = sum_k w_rk p[idx_rk].
template <typename T, int NPTS>
__device__ __forceinline__ void gather_receivers(const T* __restrict__ lvl, T* __restrict__ traces,
                                                 const int64_t* __restrict__ idx,
                                                 const T* __restrict__ w, int n_rec, int n_t, int j,
                                                 int s) {
  const long long nthr = (long long)gridDim.x * gridDim.y * blockDim.x * blockDim.y;
  for (long long r = global_thread_in_shot(); r < n_rec; r += nthr) {
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < NPTS; ++k) acc += w[r * NPTS + k] * lvl[idx[r * NPTS + k]];
    traces[((long long)s * n_rec + r) * n_t + j] = acc;
  }
}

// ------------------------------------------------------------------------------------------
// 3-D kernels: thread (tx, ty) owns (y, z) = (by*blockDim.y + ty, bz*32 + tx) and RX planes
// along x starting at x0 = blockIdx.y*RX; blockIdx.x enumerates (y-tile, z-tile).
// ------------------------------------------------------------------------------------------
struct Tile3 {
  int y, z, x0;
};
__device__ __forceinline__ Tile3 tile3(int n2, int RX) {
  const int zt = (n2 + blockDim.x - 1) / blockDim.x;
  Tile3 t;
  t.z = (blockIdx.x % zt) * blockDim.x + threadIdx.x;
  t.y = (blockIdx.x / zt) * blockDim.y + threadIdx.y;
  t.x0 = blockIdx.y * RX;
  return t;
}

template <typename T, int R, bool AB, int RX, bool ADJ>
__global__ void __launch_bounds__(256) step3d(KGrid<T> g, Step3<T> a) {
  const int s = blockIdx.z;
  const long long so = (long long)s * g.field;
  const T* __restrict__ pc = a.cur + so;
  if (!ADJ && a.traces) gather_receivers<T, 8>(pc, a.traces, a.rec_idx, a.rec_w, a.n_rec, a.n_t, a.j, s);
  const Tile3 t = tile3(g.n2, RX);
  if (t.z >= g.n2 || t.y >= g.n1 || t.x0 >= g.n0) return;
  const long long base = g.origin + (long long)t.x0 * g.s0 + (long long)t.y * g.s1 + t.z;
  T col[RX + 2 * R];
#pragma unroll
  for (int k = 0; k < RX + 2 * R; ++k) {
    const int xr = t.x0 - R + k;
    col[k] = (xr < g.n0 + R) ? pc[base + (long long)(k - R) * g.s0] : T(0);
  }
  int bx = -4, by = -4, bz = -4;
  T sw[8];
  T wn = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) sw[k] = 0;
  if (!ADJ && a.src_corner) {
    bx = a.src_corner[3 * s]; by = a.src_corner[3 * s + 1]; bz = a.src_corner[3 * s + 2];
    if (bz <= t.z && t.z <= bz + 1 && by <= t.y && t.y <= by + 1 && bx + 1 >= t.x0 && bx <= t.x0 + RX - 1) {
#pragma unroll
      for (int k = 0; k < 8; ++k) sw[k] = a.src_w[8 * s + k];
      wn = a.wavelet[a.n];
    } else {
      bx = -4;
    }
  }
  const T* __restrict__ ln = (ADJ && a.lap) ? a.lap + so : nullptr;
#pragma unroll
  for (int k = 0; k < RX; ++k) {
    const int x = t.x0 + k;
    if (x < g.n0) {
      const long long i = base + (long long)k * g.s0;
      const T c = col[k + R];
      T lap = g.wc * c + g.w1a * (col[k + R - 1] + col[k + R + 1]) +
              g.w1b * (pc[i - g.s1] + pc[i + g.s1]) + g.w1c * (pc[i - 1] + pc[i + 1]);
      if (R == 2)
        lap += g.w2a * (col[k] + col[k + 4]) + g.w2b * (pc[i - 2 * g.s1] + pc[i + 2 * g.s1]) +
               g.w2c * (pc[i - 2] + pc[i + 2]);
      const T pp = a.prev[so + i];
      T av = T(1), bv = T(1);
      bool layer = false;
      if (AB) {
        layer = x < g.lo0 || x >= g.hi0 || t.y < g.lo1 || t.y >= g.hi1 || t.z < g.lo2 || t.z >= g.hi2;
        if (layer) { av = a.A[i]; bv = (!ADJ && a.b_one) ? T(1) : a.B[i]; }
      }
      if (!ADJ && a.lap_out) a.lap_out[so + i] = lap;
      T rhs = (T(2) * c - bv * pp) + a.C[i] * lap;
      if (!ADJ) {
        const int dx = x - bx, dy = t.y - by, dz = t.z - bz;
        if (dx >= 0 && dx <= 1 && dy >= 0 && dy <= 1 && dz >= 0 && dz <= 1) rhs += sw[4 * dx + 2 * dy + dz] * wn;
      }
      a.next[so + i] = (layer && (!ADJ || a.apply_a)) ? av * rhs : rhs;
      if (ln) a.grad[so + i] += c * ln[i];
    }
  }
}

// ------------------------------------------------------------------------------------------
// Small kernels: receiver gather, adjoint injection, medium/initial-state preparation,
// gradient reduction and the snapshot codec.
// ------------------------------------------------------------------------------------------
template <typename T, int NPTS>
__global__ void sample_kernel(const T* __restrict__ lvl, long long field, T* __restrict__ traces,
                              const int64_t* __restrict__ idx, const T* __restrict__ w, int n_rec,
                              int n_t, int j) {
  const int s = blockIdx.y;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rec) return;
  const T* p = lvl + (long long)s * field;
  T acc = T(0);
#pragma unroll
  for (int k = 0; k < NPTS; ++k) acc += w[(long long)r * NPTS + k] * p[idx[(long long)r * NPTS + k]];
  traces[((long long)s * n_rec + r) * n_t + j] = acc;
}

// out[s][cell] += (apply_a ? A[cell] : 1) * C[cell] * sum_e w_e g[s, rec_e, j], cells in CSR order
// (the adjoint source of q = C mu).
template <typename T>
__global__ void inject_kernel(T* __restrict__ out, long long field, const T* __restrict__ C, const T* __restrict__ A,
                              int apply_a, const T* __restrict__ g, int n_rec, int n_t, int j,
                              int n_cells, const int64_t* __restrict__ cell,
                              const int* __restrict__ ptr, const int* __restrict__ rec,
                              const T* __restrict__ w) {
  const int s = blockIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  T acc = T(0);
  const T* gs = g + (long long)s * n_rec * n_t + j;
  for (int e = ptr[c]; e < ptr[c + 1]; ++e) acc += w[e] * gs[(long long)rec[e] * n_t];
  const long long i = cell[c];
  const T av = (apply_a && A) ? A[i] : T(1);
  out[(long long)s * field + i] += av * (C[i] * acc);
}

}  // namespace nw
