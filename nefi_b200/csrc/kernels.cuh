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

// Programmatic dependent launch: block until the preceding grid's memory is visible / allow the
// following grid to be scheduled. Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void wait_previous_grid() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void allow_next_grid() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

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

// Receiver gather of one level for shot s by the `nthr` threads of the launch that work on that shot
// (this thread is number `thr` of them): traces[s, r, j] = sum_k w_rk p[idx_rk].
template <typename T, int NPTS>
__device__ __forceinline__ void gather_receivers(const T* __restrict__ lvl, T* __restrict__ traces,
                                                 const int64_t* __restrict__ idx,
                                                 const T* __restrict__ w, int n_rec, int n_t, int j,
                                                 int s, long long thr, long long nthr) {
  for (long long r = thr; r < n_rec; r += nthr) {
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < NPTS; ++k) acc += w[r * NPTS + k] * lvl[idx[r * NPTS + k]];
    traces[((long long)s * n_rec + r) * n_t + j] = acc;
  }
}

// ------------------------------------------------------------------------------------------
// Small kernels: receiver gather, adjoint injection, medium/initial-state preparation,
// gradient reduction and the snapshot codec.
// ------------------------------------------------------------------------------------------
// The sample of receiver r in the field p (its NPTS stencil points, in table order).
template <typename T, int NPTS>
__device__ __forceinline__ T sample_point(const T* __restrict__ p, const int64_t* __restrict__ idx,
                                          const T* __restrict__ w, int r) {
  T acc = T(0);
#pragma unroll
  for (int k = 0; k < NPTS; ++k) acc += w[(long long)r * NPTS + k] * p[idx[(long long)r * NPTS + k]];
  return acc;
}

template <typename T, int NPTS>
__global__ void sample_kernel(const T* __restrict__ lvl, long long field, T* __restrict__ traces,
                              const int64_t* __restrict__ idx, const T* __restrict__ w, int n_rec,
                              int n_t, int j) {
  wait_previous_grid();
  allow_next_grid();
  const int s = blockIdx.y;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rec) return;
  traces[((long long)s * n_rec + r) * n_t + j] = sample_point<T, NPTS>(lvl + (long long)s * field, idx, w, r);
}

// out[s][cell] += (apply_a ? A[cell] : 1) * C[cell] * sum_e w_e g[s, rec_e, j], cells in CSR order
// (the adjoint source of q = C mu).
template <typename T>
__global__ void inject_kernel(T* __restrict__ out, long long field, const T* __restrict__ C, const T* __restrict__ A,
                              int apply_a, const T* __restrict__ g, int n_rec, int n_t, int j,
                              int n_cells, const int64_t* __restrict__ cell,
                              const int* __restrict__ ptr, const int* __restrict__ rec,
                              const T* __restrict__ w) {
  wait_previous_grid();
  allow_next_grid();
  const int s = blockIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  T acc = T(0);
  const T* gs = g + (long long)s * n_rec * n_t + j;
  for (int e = ptr[c]; e < ptr[c + 1]; ++e) acc = fma_rn(w[e], gs[(long long)rec[e] * n_t], acc);
  const long long i = cell[c];
  const T av = (apply_a && A) ? A[i] : T(1);
  T* o = out + (long long)s * field + i;
  *o = fma_rn(av, mul_rn(C[i], acc), *o);  // the rounding sequence of the PML layer launch's own injection
}

}  // namespace nw
