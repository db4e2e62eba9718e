// stencil2d.cuh — tiled 2-D leapfrog kernels for sm_100a.
//
// One CTA (8 warps) owns a tile of TX = 8*RX rows by TZ = 32*VZ columns and loops over a group
// of shots; the hardware scheduler balances the (tile, shot group) CTAs over the SMs, which
// absorbs the extra cost of tiles in the absorbing layer. A thread owns VZ adjacent columns and
// RX rows: it slides a (2R+1)-row register window down its columns, reading each row of the
// stencil field once as a VZ-wide vector plus two halo vectors from shared memory, so every
// shared-memory access is a conflict-free 8- or 16-byte load. The stencil field (p^n, or q^{n+1}
// in the adjoint) is staged per shot with an R-row and 16-byte-column halo by cp.async through a
// ring of NS buffers, so the copies of the next NS-1 shots are in flight while shot s is computed.
// Each thread computes the shared/global offsets of the 16-byte chunks it copies once per CTA;
// per shot it only adds the shot's base address.
//
// The two directions feed the per-cell fields differently, each the faster way on a 552^2 grid:
//  - fwd2d stages c^2 dt^2 and (in absorbing-layer tiles) A and B once per CTA and loads p^{n-1},
//    which it reads only at its own cells, straight into registers one shot ahead of its use;
//  - adj2d stages q^{n+2} and the stored Lap p^n as core tiles in the same cp.async ring, and
//    c^2 dt^2, A, B (layer tiles) and its group's gradient accumulator tile once per CTA, which
//    keeps its register count at three CTAs per SM next to the gradient sums it holds.
//
// The step kernels are launched with programmatic dependent launch: each one waits
// (griddepcontrol.wait) for the previous kernel in the stream to finish and flush before it reads
// or writes any field, and lets the next one be scheduled (griddepcontrol.launch_dependents) as
// soon as its own last wave is resident, which hides the launch gap between time steps.
//
// Receivers are gathered and adjoint sources injected inside the same kernels, from per-tile
// tables built on the host (the receivers whose stencil corner lies in the tile; the cells of the
// tile that receiver stencils touch), in a fixed order, and the stencil arithmetic has a fixed
// rounding sequence (fma_rn and friends), so results are bitwise reproducible and independent of
// the tile shape.
#pragma once
#include <type_traits>

#include "kernels.cuh"

namespace nw {

__device__ __forceinline__ void cp_async16(unsigned smem, const void* gmem) {  // smem: shared-window address
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Vector of N elements of T loaded/stored as one 8- or 16-byte access.
template <typename T, int N>
__device__ __forceinline__ void vload(const T* p, T (&o)[N]) {
  static_assert(sizeof(T) * N == 8 || sizeof(T) * N == 16, "vector width");
  if constexpr (sizeof(T) * N == 16) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    const T* q = reinterpret_cast<const T*>(&t);
#pragma unroll
    for (int i = 0; i < N; ++i) o[i] = q[i];
  } else {
    const float2 t = *reinterpret_cast<const float2*>(p);
    const T* q = reinterpret_cast<const T*>(&t);
#pragma unroll
    for (int i = 0; i < N; ++i) o[i] = q[i];
  }
}
// Read-only global load through the non-coherent (L1) path.
template <typename T, int N>
__device__ __forceinline__ void vldg(const T* p, T (&o)[N]) {
  if constexpr (sizeof(T) * N == 16) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    const T* q = reinterpret_cast<const T*>(&t);
#pragma unroll
    for (int i = 0; i < N; ++i) o[i] = q[i];
  } else {
    const float2 t = __ldg(reinterpret_cast<const float2*>(p));
    const T* q = reinterpret_cast<const T*>(&t);
#pragma unroll
    for (int i = 0; i < N; ++i) o[i] = q[i];
  }
}
// Global load through L2 only (ld.global.cg): used for levels an earlier kernel wrote, read before
// griddepcontrol.wait, where a line left in this SM's L1 by an older kernel must not be returned.
template <typename T, int N>
__device__ __forceinline__ void vldcg(const T* p, T (&o)[N]) {
  if constexpr (sizeof(T) * N == 16) {
    const float4 t = __ldcg(reinterpret_cast<const float4*>(p));
    const T* q = reinterpret_cast<const T*>(&t);
#pragma unroll
    for (int i = 0; i < N; ++i) o[i] = q[i];
  } else {
    const float2 t = __ldcg(reinterpret_cast<const float2*>(p));
    const T* q = reinterpret_cast<const T*>(&t);
#pragma unroll
    for (int i = 0; i < N; ++i) o[i] = q[i];
  }
}
template <typename T, int N>
__device__ __forceinline__ void vstore(T* p, const T (&o)[N]) {
  if constexpr (sizeof(T) * N == 16) {
    float4 t;
    T* q = reinterpret_cast<T*>(&t);
#pragma unroll
    for (int i = 0; i < N; ++i) q[i] = o[i];
    *reinterpret_cast<float4*>(p) = t;
  } else {
    float2 t;
    T* q = reinterpret_cast<T*>(&t);
#pragma unroll
    for (int i = 0; i < N; ++i) q[i] = o[i];
    *reinterpret_cast<float2*>(p) = t;
  }
}

// Per-tile tables, built on the host for one tile shape (TX, TZ).
struct TileTables {
  int tiles_z;                        // tiles along the contiguous axis (gridDim.x)
  const int* __restrict__ rec_ptr;    // (n_tiles + 1): receivers whose stencil corner is in the tile
  const int* __restrict__ rec_list;   // receiver ids
  const int* __restrict__ rec_corner; // (n_rec, 2) corner cell (x, z)
  const int* __restrict__ cell_ptr;   // (n_tiles + 1): receiver-touched cells of the tile
  const int* __restrict__ cell_local; // (x - x0) * TZ + (z - z0)
  const int* __restrict__ cell_gid;   // row of the cell in the global cell table
  const int* __restrict__ gcell_ptr;  // global cell table: entries of each touched cell
  const int* __restrict__ gcell_rec;
};

// Everything one tiled step reads and writes. The forward step advances the pressure,
//   p^{n+1} = A (2 p^n - B p^{n-1} + C Lap p^n + S w(n)),
// and the adjoint step advances q = C mu (mu^n = A lambda^n), which obeys the same recursion,
//   q^n = A (2 q^{n+1} - B q^{n+2} + C Lap q^{n+1} + C R^T g_n),
// so both directions run the same stencil: multiplying the adjoint of the reference's scheme,
// mu^n = A (R^T g_n + 2 mu^{n+1} + Lap(C mu^{n+1}) - B mu^{n+2}), by C moves C out of the Laplacian.
// The velocity gradient sum_n mu^{n+1} Lap p^n is accumulated as sum_n q^{n+1} Lap p^n, i.e. C dJ/dC.
template <typename T>
struct Tiled2 {
  const T* __restrict__ prev;   // forward p^{n-1}   | adjoint q^{n+2}  (core tiles)
  const T* __restrict__ cur;    // forward p^n       | adjoint q^{n+1}  (halo tiles)
  T* __restrict__ next;         // forward p^{n+1}   | adjoint q^n
  const T* __restrict__ C;
  const T* __restrict__ A;
  const T* __restrict__ B;
  int b_one;                    // forward: B = 1 on the first step (Cerjan)
  int prev_ready;               // forward: p^{n-1} was written two or more launches back, so it may be
                                // read before griddepcontrol.wait (0: after it)
  int apply_a;                  // adjoint: A applies (n >= 1); at n = 0 the output is C lambda^0
  int lap_ready;                // adjoint: Lap p^n was written two or more launches back, so its tiles
                                // may be copied before griddepcontrol.wait (q^{n+2} always may: the
                                // adjoint step two launches back wrote it)
  int n_shots, shots_per_cta;
  // forward: point sources, receiver samples of p^n
  const int* __restrict__ src_corner;
  const T* __restrict__ src_w;
  const T* __restrict__ wavelet;
  int n;
  T* __restrict__ traces;       // non-null on record steps
  const T* __restrict__ rec_w;
  T* __restrict__ lap_out;      // non-null: also store Lap p^n (the gradient factor)
  // adjoint: receiver injection and the gradient
  const T* __restrict__ gtr;    // trace cotangents (n_shots, n_rec, n_t); non-null on record steps
  const T* __restrict__ gcell_w;
  const T* __restrict__ lap;    // Lap p^n as the forward step stored it; nullptr: no gradient term
  T* __restrict__ gacc;         // (n_groups, field) accumulators of C dJ/dC, one per shot group
  int n_rec, n_t, j;
  TileTables tt;
  // the cells a launch steps: tiles start at (tx_off, tz_off) (tz_off a multiple of the 16-byte chunk)
  // and only cells below (x_end, z_end) are stored; the whole grid is (0, 0, n0, n1), a sub-box is the
  // PML's interior
  int tx_off, tz_off, x_end, z_end;
  // two steps per launch (fwd2t): the second step's outputs p^{n+2} and Lap p^{n+1}, and its receiver
  // samples of level n+1 (traces1 non-null on record steps, sample j1); two = 0: the first step only
  int two;
  T* __restrict__ next2;
  T* __restrict__ lap_out1;
  T* __restrict__ traces1;
  int j1;
};

template <typename T, int VZ, int RX, int R>
struct Tile2Shape {
  static constexpr int TZ = 32 * VZ;
  static constexpr int TX = 8 * RX;
  static constexpr int HL = 16 / (int)sizeof(T);  // halo columns per side (one 16-byte chunk)
  static constexpr int SW = TZ + 2 * HL;          // shared row width of halo tiles
  static constexpr int EPC = 16 / (int)sizeof(T); // elements per 16-byte chunk
  static constexpr int HR = TX + 2 * R;           // rows of a halo tile
  static constexpr int PS = HR * SW;              // elements of a halo tile
  static constexpr int QS = TX * TZ;              // elements of a core tile
  static constexpr int NCH = (HR * (SW / EPC) + 255) / 256;  // halo chunks per thread
  static constexpr int NCC = (TX * (TZ / EPC) + 255) / 256;  // core chunks per thread
  static constexpr int NS = sizeof(T) == 8 ? 2 : 3;          // shot buffers in the copy ring
  // the adjoint stages three tiles per shot: a two-shot ring keeps larger tiles at 3 CTAs per SM
  static constexpr int NSA = (sizeof(T) == 8 || RX >= 4) ? 2 : 3;
};

// The chunks one thread copies for one tile region: the shared byte offset in the destination tile
// and the global element offset relative to a field's base (-1 marks a chunk outside the stored rows).
template <int NC>
struct CopyPlan {
  unsigned soff[NC];
  int goff[NC];
};

// Halo tile: rows [x0 - R, x0 + TX + R) x columns [z0 - HL, z0 + TZ + HL), row pitch SW.
// Rows past the last ghost row and chunks past the row pitch are not stored.
template <typename T, int VZ, int RX, int R>
__device__ __forceinline__ CopyPlan<Tile2Shape<T, VZ, RX, R>::NCH> plan_halo(const KGrid<T>& g, int x0, int z0) {
  using S = Tile2Shape<T, VZ, RX, R>;
  constexpr int CPR = S::SW / S::EPC;
  CopyPlan<S::NCH> p;
#pragma unroll
  for (int i = 0; i < S::NCH; ++i) {
    const int c = threadIdx.x + 256 * i;
    const int row = c / CPR, ch = c - row * CPR;
    const int x = x0 - R + row;
    const int z = z0 - S::HL + ch * S::EPC;
    p.soff[i] = (unsigned)((row * S::SW + ch * S::EPC) * sizeof(T));
    p.goff[i] = (c < S::HR * CPR && x >= -R && x < g.n0 + R && z < (int)g.s0)
                    ? (int)(g.origin + (long long)x * g.s0 + z) : -1;
  }
  return p;
}
// Core tile: rows [x0, x0 + TX) x columns [z0, z0 + TZ), row pitch TZ.
template <typename T, int VZ, int RX, int R>
__device__ __forceinline__ CopyPlan<Tile2Shape<T, VZ, RX, R>::NCC> plan_core(const KGrid<T>& g, int x0, int z0) {
  using S = Tile2Shape<T, VZ, RX, R>;
  constexpr int CPR = S::TZ / S::EPC;
  CopyPlan<S::NCC> p;
#pragma unroll
  for (int i = 0; i < S::NCC; ++i) {
    const int c = threadIdx.x + 256 * i;
    const int row = c / CPR, ch = c - row * CPR;
    const int x = x0 + row;
    const int z = z0 + ch * S::EPC;
    p.soff[i] = (unsigned)((row * S::TZ + ch * S::EPC) * sizeof(T));
    p.goff[i] = (c < S::TX * CPR && x < g.n0 && z < (int)g.s0) ? (int)(g.origin + (long long)x * g.s0 + z) : -1;
  }
  return p;
}
// Shared-window address of a shared-memory pointer.
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
// Issues one thread's chunks of a tile: field is the global field, dst the tile's shared-window address.
template <typename T, int NC>
__device__ __forceinline__ void issue(const CopyPlan<NC>& p, const T* __restrict__ field, unsigned dst) {
#pragma unroll
  for (int i = 0; i < NC; ++i)
    if (p.goff[i] >= 0) cp_async16(dst + p.soff[i], field + p.goff[i]);
}

// Row loader of the sliding window: own VZ vector and the two neighbouring vectors.
template <typename T, int VZ>
struct Row3 {
  T l[VZ], c[VZ], r[VZ];
};
template <typename T, int VZ>
__device__ __forceinline__ T zval(const Row3<T, VZ>& w, int u) {  // column u in [-VZ, 2VZ)
  return u < 0 ? w.l[VZ + u] : (u >= VZ ? w.r[u - VZ] : w.c[u]);
}

template <typename T, int VZ>
__device__ __forceinline__ void store_row(T* dst, const T (&o)[VZ], int zc, int n1) {
  if (zc + VZ <= n1) {
    vstore<T, VZ>(dst, o);
  } else {
#pragma unroll
    for (int v = 0; v < VZ; ++v)
      if (zc + v < n1) dst[v] = o[v];
  }
}


// The Laplacian of the window's centre row at column v, and the leapfrog update, in a fixed
// rounding sequence.
template <typename T, int R, int VZ>
__device__ __forceinline__ T lap_at(const T (&wv)[2 * R + 1][VZ], const Row3<T, VZ>& rw, int v, T wc, T w1x,
                                    T w1z, T w2x, T w2z) {
  T lap = fma_rn(w1z, add_rn(zval(rw, v - 1), zval(rw, v + 1)),
                 fma_rn(w1x, add_rn(wv[R - 1][v], wv[R + 1][v]), mul_rn(wc, wv[R][v])));
  if (R == 2)
    lap = fma_rn(w2z, add_rn(zval(rw, v - 2), zval(rw, v + 2)), fma_rn(w2x, add_rn(wv[0][v], wv[4][v]), lap));
  return lap;
}

// ------------------------------------------------------------------------------------------
// Forward step of every shot of a group over one tile: p^{n+1} = A (2 p^n - B p^{n-1} +
// C Lap p^n + S w(n)); also samples the tile's receivers from the staged p^n tile, adds the
// shots' point sources and, with lap_out, stores Lap p^n (the gradient factor).
// ------------------------------------------------------------------------------------------
template <typename T, int R, int VZ, int RX, bool AB>
__device__ __forceinline__ void fwd2d_body(const KGrid<T>& g, const Tiled2<T>& a, int bx, int by, int bz,
                                           unsigned char* smem_raw) {
  using S = Tile2Shape<T, VZ, RX, R>;
  constexpr int NS = S::NS;
  T* scc = reinterpret_cast<T*>(smem_raw);  // [QS] C
  T* sa = scc + S::QS;                      // [QS] A (layer tiles)
  T* sbb = sa + S::QS;                      // [QS] B (layer tiles)
  T* sp = sbb + S::QS;                      // [NS][PS] p^n with halo

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int z0 = bx * S::TZ + a.tz_off, x0 = by * S::TX + a.tx_off;
  const int tile = by * a.tt.tiles_z + bx;
  const int sb = bz * a.shots_per_cta;
  const int se = min(sb + a.shots_per_cta, a.n_shots);
  const int zc = z0 + lane * VZ;  // first owned column
  const int xr = x0 + warp * RX;  // first owned row
  const int lrow = warp * RX;     // first owned row inside the tile
  const bool own_cols = zc < a.z_end;
  const int ld = (int)g.s0;
  const long long cbase = g.origin + (long long)xr * ld + zc;  // owned cells of row k: + k*ld
  bool ok[RX];  // row k of the owned cells lies in the grid
#pragma unroll
  for (int k = 0; k < RX; ++k) ok[k] = own_cols && xr + k < a.x_end;

  const bool layer_tile = AB && (x0 < g.lo0 || x0 + S::TX > g.hi0 || z0 < g.lo1 || z0 + S::TZ > g.hi1);
  const bool use_b = layer_tile && !a.b_one;
  const CopyPlan<S::NCH> ph = plan_halo<T, VZ, RX, R>(g, x0, z0);
  const CopyPlan<S::NCC> pc = plan_core<T, VZ, RX, R>(g, x0, z0);
  // Before the wait, while the previous step finishes: everything this launch reads that no kernel
  // still running writes -- the coefficients (constant over the sweep), the per-tile tables, the
  // first shot's source corner, and p^{n-1}, which the step two launches back wrote (that launch
  // completed before the previous one passed its own wait, which had to happen before this one
  // could start) and which nothing writes until this step has finished reading it.
  constexpr unsigned PSB = S::PS * sizeof(T);  // bytes of one halo tile of the ring
  const unsigned sp_s = smem_addr(sp);
  issue(pc, a.C, smem_addr(scc));  // once per CTA, in the first commit group
  if (layer_tile) {
    issue(pc, a.A, smem_addr(sa));
    issue(pc, a.B, smem_addr(sbb));
  }
  T pv[RX][VZ];  // p^{n-1} of the owned cells, one shot ahead
#pragma unroll
  for (int k = 0; k < RX; ++k) {
#pragma unroll
    for (int v = 0; v < VZ; ++v) pv[k][v] = T(0);
    if (a.prev_ready && ok[k]) vldcg<T, VZ>(a.prev + (long long)sb * g.field + cbase + (long long)k * ld, pv[k]);
  }
  int e0 = 0, e1 = 0;
  if (a.traces) { e0 = a.tt.rec_ptr[tile]; e1 = a.tt.rec_ptr[tile + 1]; }
  // thread t samples the tile's receiver e0 + t: its id and staged-tile offset, read once per CTA
  // (receivers past the first 256 of the tile read theirs every shot)
  int rr = -1, roff = 0;
  if (e0 + (int)threadIdx.x < e1) {
    rr = a.tt.rec_list[e0 + threadIdx.x];
    roff = (a.tt.rec_corner[2 * rr] - x0 + R) * S::SW + a.tt.rec_corner[2 * rr + 1] - z0 + S::HL;
  }
  int2 scor = make_int2(-1 << 20, -1 << 20);  // the next shot's source corner (x, z), one shot ahead
  if (a.src_corner) scor = make_int2(a.src_corner[2 * sb], a.src_corner[2 * sb + 1]);
  wait_previous_grid();
  allow_next_grid();
  if (!a.prev_ready) {  // p^{n-1} came from the launch just before (a snapshot decode, an initial state)
#pragma unroll
    for (int k = 0; k < RX; ++k)
      if (ok[k]) vldg<T, VZ>(a.prev + (long long)sb * g.field + cbase + (long long)k * ld, pv[k]);
  }
#pragma unroll
  for (int i = 0; i < NS - 1; ++i) {  // one commit group per shot, empty groups included, so that
    if (sb + i < se) issue(ph, a.cur + (long long)(sb + i) * g.field, sp_s + i * PSB);
    cp_async_commit();                // wait_group<NS-1> in the loop means "shot s has landed"
  }
  const T wc = g.wc, w1x = g.w1a, w1z = g.w1b, w2x = g.w2a, w2z = g.w2b;

  // running per-shot state: the ring buffer of shot s, and the fields of shot s (stores), s + 1
  // (p^{n-1} prefetch) and s + NS - 1 (the halo copy issued during shot s)
  const long long fs = g.field;
  int buf = 0;
  const T* gcopy = a.cur + (long long)(sb + NS - 1) * fs;
  T* nxt = a.next + (long long)sb * fs + cbase;
  T* lpo = a.lap_out ? a.lap_out + (long long)sb * fs + cbase : nullptr;
  const T* pvn = a.prev + (long long)sb * fs + cbase;  // advanced to shot s + 1 before use
  for (int s = sb; s < se; ++s) {
    cp_async_wait<NS - 2>();  // this thread's copies of shot s have landed
    __syncthreads();          // everyone's have, and every thread is done with shot s-1
    {
      const int nb = buf == 0 ? NS - 1 : buf - 1;  // the buffer shot s-1 used
      if (s + NS - 1 < se) issue(ph, gcopy, sp_s + nb * PSB);
      cp_async_commit();
      gcopy += fs;
    }
    const T* P = sp + buf * S::PS;
    pvn += fs;

    if (rr >= 0) {  // receiver samples of p^n
      const T* w = a.rec_w + 4 * rr;
      T acc = mul_rn(w[0], P[roff]);
      acc = fma_rn(w[1], P[roff + 1], acc);
      acc = fma_rn(w[2], P[roff + S::SW], acc);
      acc = fma_rn(w[3], P[roff + S::SW + 1], acc);
      a.traces[((long long)s * a.n_rec + rr) * a.n_t + a.j] = acc;
    }
    for (int e = e0 + threadIdx.x + 256; e < e1; e += 256) {  // the tile's receivers past the first 256
      const int r = a.tt.rec_list[e];
      const int row = a.tt.rec_corner[2 * r] - x0 + R, col = a.tt.rec_corner[2 * r + 1] - z0 + S::HL;
      const T* w = a.rec_w + 4 * r;
      T acc = mul_rn(w[0], P[row * S::SW + col]);
      acc = fma_rn(w[1], P[row * S::SW + col + 1], acc);
      acc = fma_rn(w[2], P[(row + 1) * S::SW + col], acc);
      acc = fma_rn(w[3], P[(row + 1) * S::SW + col + 1], acc);
      a.traces[((long long)s * a.n_rec + r) * a.n_t + a.j] = acc;
    }
    // the shot's source stencil, if it touches this tile (a CTA-uniform test)
    bool src_tile = false;
    T sw0 = 0, sw1 = 0, sw2 = 0, sw3 = 0;
    const int bx = scor.x, bz = scor.y;
    if (a.src_corner) {
      if (s + 1 < se) scor = make_int2(a.src_corner[2 * (s + 1)], a.src_corner[2 * (s + 1) + 1]);
      src_tile = bx + 1 >= x0 && bx < x0 + S::TX && bz + 1 >= z0 && bz < z0 + S::TZ;
      if (src_tile) {
        const T wn = a.wavelet[a.n];
        sw0 = mul_rn(a.src_w[4 * s], wn); sw1 = mul_rn(a.src_w[4 * s + 1], wn);
        sw2 = mul_rn(a.src_w[4 * s + 2], wn); sw3 = mul_rn(a.src_w[4 * s + 3], wn);
      }
    }
    const bool more = s + 1 < se;

    // sliding window: wv[q] holds tile row (lrow + k + q - R) (own columns only)
    T wv[2 * R + 1][VZ];
#pragma unroll
    for (int q = 0; q < 2 * R; ++q) vload<T, VZ>(P + (lrow + q) * S::SW + S::HL + lane * VZ, wv[q]);
#pragma unroll
    for (int k = 0; k < RX; ++k) {
      const int prow = lrow + k + R;  // shared row of the output row
      vload<T, VZ>(P + (prow + R) * S::SW + S::HL + lane * VZ, wv[2 * R]);
      Row3<T, VZ> rw;
      vload<T, VZ>(P + prow * S::SW + S::HL + lane * VZ - VZ, rw.l);
#pragma unroll
      for (int v = 0; v < VZ; ++v) rw.c[v] = wv[R][v];
      vload<T, VZ>(P + prow * S::SW + S::HL + lane * VZ + VZ, rw.r);
      const int x = xr + k;
      const int toff = (lrow + k) * S::TZ + lane * VZ;  // the owned cells in a core tile
      T cc[VZ], ca[VZ], cb[VZ];
      vload<T, VZ>(scc + toff, cc);
#pragma unroll
      for (int v = 0; v < VZ; ++v) { ca[v] = T(1); cb[v] = T(1); }
      if (layer_tile) vload<T, VZ>(sa + toff, ca);
      if (use_b) vload<T, VZ>(sbb + toff, cb);
      T o[VZ], lp[VZ];
#pragma unroll
      for (int v = 0; v < VZ; ++v) {
        lp[v] = lap_at<T, R, VZ>(wv, rw, v, wc, w1x, w1z, w2x, w2z);
        o[v] = fma_rn(cc[v], lp[v], fma_rn(-cb[v], pv[k][v], add_rn(wv[R][v], wv[R][v])));
      }
      if (src_tile) {
#pragma unroll
        for (int v = 0; v < VZ; ++v) {
          const int dx = x - bx, dz = zc + v - bz;
          if (dx >= 0 && dx <= 1 && dz >= 0 && dz <= 1)
            o[v] = add_rn(o[v], (dx == 0) ? (dz == 0 ? sw0 : sw1) : (dz == 0 ? sw2 : sw3));
        }
      }
      if (layer_tile) {
#pragma unroll
        for (int v = 0; v < VZ; ++v) o[v] = mul_rn(ca[v], o[v]);
      }
      if (ok[k]) {
        store_row<T, VZ>(nxt + k * ld, o, zc, a.z_end);
        if (lpo) store_row<T, VZ>(lpo + k * ld, lp, zc, a.z_end);
        if (more) vldg<T, VZ>(pvn + k * ld, pv[k]);  // in flight while the rest of this shot runs
      }
#pragma unroll
      for (int q = 0; q < 2 * R; ++q)
#pragma unroll
        for (int v = 0; v < VZ; ++v) wv[q][v] = wv[q + 1][v];
    }
    nxt += fs;
    if (lpo) lpo += fs;
    buf = buf + 1 == NS ? 0 : buf + 1;
  }
}

// ------------------------------------------------------------------------------------------
// Adjoint step of every shot of a group over one tile: q^n = A (2 q^{n+1} - B q^{n+2} +
// C (Lap q^{n+1} + R^T g_n)), with the receiver cotangents injected at the touched cells of the
// tile; accumulates q^{n+1} Lap p^n over the group's shots in registers and adds the sum into
// the group's accumulator (one writer per cell and group).
// ------------------------------------------------------------------------------------------
template <typename T, int R, int VZ, int RX, bool AB>
__device__ __forceinline__ void adj2d_body(const KGrid<T>& g, const Tiled2<T>& a, int bx, int by, int bz,
                                           unsigned char* smem_raw) {
  using S = Tile2Shape<T, VZ, RX, R>;
  constexpr int NS = S::NSA;
  T* scc = reinterpret_cast<T*>(smem_raw);  // [QS] C
  T* sa = scc + S::QS;                      // [QS] A (layer tiles)
  T* sbb = sa + S::QS;                      // [QS] B (layer tiles)
  T* sg = sbb + S::QS;                      // [QS] the group's gradient accumulator
  T* sp = sg + S::QS;                       // [NS][PS] q^{n+1} with halo
  T* sq = sp + NS * S::PS;                  // [NS][QS] q^{n+2}
  T* sl = sq + NS * S::QS;                  // [NS][QS] Lap p^n
  T* sj = sl + NS * S::QS;                  // [2][QS] cotangents injected at a shot's cells, by shot parity

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int z0 = bx * S::TZ + a.tz_off, x0 = by * S::TX + a.tx_off;
  const int tile = by * a.tt.tiles_z + bx;
  const int sb = bz * a.shots_per_cta;
  const int se = min(sb + a.shots_per_cta, a.n_shots);
  const int zc = z0 + lane * VZ;  // first owned column
  const int xr = x0 + warp * RX;  // first owned row
  const int lrow = warp * RX;     // first owned row inside the tile
  const bool own_cols = zc < a.z_end;
  const bool grad = a.lap != nullptr;

  const bool layer_tile = AB && (x0 < g.lo0 || x0 + S::TX > g.hi0 || z0 < g.lo1 || z0 + S::TZ > g.hi1);
  const CopyPlan<S::NCH> ph = plan_halo<T, VZ, RX, R>(g, x0, z0);
  const CopyPlan<S::NCC> pc = plan_core<T, VZ, RX, R>(g, x0, z0);
  // once per CTA, in the first commit group: C, A and B (layer tiles), constant over the sweep, so
  // issued before the wait while the previous step finishes
  constexpr unsigned PSB = S::PS * sizeof(T), QSB = S::QS * sizeof(T);  // bytes of a halo / core tile
  const unsigned sp_s = smem_addr(sp), sq_s = smem_addr(sq), sl_s = smem_addr(sl);
  issue(pc, a.C, smem_addr(scc));
  if (layer_tile) {
    issue(pc, a.A, smem_addr(sa));
    issue(pc, a.B, smem_addr(sbb));
  }
  int c0 = 0, c1 = 0;
  if (a.gtr) { c0 = a.tt.cell_ptr[tile]; c1 = a.tt.cell_ptr[tile + 1]; }
  const bool inject = c1 > c0;  // uniform
  // thread t owns touched cell c0 + t of the tile; its table entries (receiver, weight) are
  // shot-independent and cached here, so a shot only loads the cotangents themselves
  constexpr int kEnt = 4;
  int jl = -1, jn = 0, jrec[kEnt];
  T jw[kEnt], jv[kEnt];  // jv: the cached entries' cotangents of the current shot, loaded one shot ahead
  bool jslow = false;  // more entries than cached: read the table every shot
  if (inject) {
    for (int i = threadIdx.x; i < 2 * S::QS; i += 256) sj[i] = T(0);
    const int e = c0 + threadIdx.x;
    if (e < c1) {
      jl = a.tt.cell_local[e];
      const int gid = a.tt.cell_gid[e];
      const int q0 = a.tt.gcell_ptr[gid];
      jn = a.tt.gcell_ptr[gid + 1] - q0;
      jslow = jn > kEnt;
#pragma unroll
      for (int m = 0; m < kEnt; ++m) {
        jrec[m] = (m < jn) ? a.tt.gcell_rec[q0 + m] : 0;
        jw[m] = (m < jn) ? a.gcell_w[q0 + m] : T(0);
      }
    }
    __syncthreads();  // zeroing completes before any thread writes a cotangent value
  }
  // the first shots' q^{n+2} core tiles (and Lap p^n, when it was not written by the launch just
  // before) join the copies issued before the wait; they land in the first commit group
#pragma unroll
  for (int i = 0; i < NS - 1; ++i)
    if (sb + i < se) {
      issue(pc, a.prev + (long long)(sb + i) * g.field, sq_s + i * QSB);
      if (grad && a.lap_ready) issue(pc, a.lap + (long long)(sb + i) * g.field, sl_s + i * QSB);
    }
  wait_previous_grid();
  allow_next_grid();
  if (jl >= 0 && !jslow) {  // the first shot's cotangents (the launch just before may have written them)
    const T* gs = a.gtr + (long long)sb * a.n_rec * a.n_t + a.j;
#pragma unroll
    for (int m = 0; m < kEnt; ++m) jv[m] = (m < jn) ? gs[(long long)jrec[m] * a.n_t] : T(0);
  }
  if (grad) issue(pc, a.gacc + (long long)bz * g.field, smem_addr(sg));  // the previous step updated it
#pragma unroll
  for (int i = 0; i < NS - 1; ++i) {  // one commit group per shot, empty groups included, so that
    if (sb + i < se) {                // wait_group<NS-1> in the loop means "shot s has landed"
      issue(ph, a.cur + (long long)(sb + i) * g.field, sp_s + i * PSB);
      if (grad && !a.lap_ready) issue(pc, a.lap + (long long)(sb + i) * g.field, sl_s + i * QSB);
    }
    cp_async_commit();
  }

  const bool use_a = layer_tile && a.apply_a;
  const T wc = g.wc, w1x = g.w1a, w1z = g.w1b, w2x = g.w2a, w2z = g.w2b;
  const int ld = (int)g.s0;
  const long long cbase = g.origin + (long long)xr * ld + zc;  // owned cells of row k: + k*ld
  T gsum[RX][VZ];  // per-cell sum over this CTA's shots
#pragma unroll
  for (int k = 0; k < RX; ++k)
#pragma unroll
    for (int v = 0; v < VZ; ++v) gsum[k][v] = T(0);

  // running per-shot state: the ring buffer of shot s, the output of shot s and the fields of shot
  // s + NS - 1, whose copies are issued during shot s
  const long long fs = g.field;
  int buf = 0;
  const long long cofs = (long long)(sb + NS - 1) * fs;
  const T* gcur = a.cur + cofs;
  const T* gprev = a.prev + cofs;
  const T* glap = grad ? a.lap + cofs : gprev;  // (not read without a gradient)
  T* ob = a.next + (long long)sb * fs + cbase;
  bool okr[RX];  // row k of the owned cells lies in the grid
#pragma unroll
  for (int k = 0; k < RX; ++k) okr[k] = own_cols && xr + k < a.x_end;
  for (int s = sb; s < se; ++s) {
    // this shot's cotangent half; shot s-2 read it last, and every thread finished shot s-2 before
    // the previous barrier, so it is free; the same thread sets the same cells every shot
    T* sjs = sj + ((s - sb) & 1) * S::QS;
    cp_async_wait<NS - 2>();  // this thread's copies of shot s have landed
    if (inject) {  // cotangent of shot s at each touched cell, summed in table order
      const T* gs = a.gtr + (long long)s * a.n_rec * a.n_t + a.j;
      if (jl >= 0 && !jslow) {
        T acc = T(0);
#pragma unroll
        for (int m = 0; m < kEnt; ++m)
          if (m < jn) acc = fma_rn(jw[m], jv[m], acc);
        sjs[jl] = acc;
        if (s + 1 < se) {  // the next shot's, in flight while this shot is computed
          const T* gn = gs + (long long)a.n_rec * a.n_t;
#pragma unroll
          for (int m = 0; m < kEnt; ++m)
            if (m < jn) jv[m] = gn[(long long)jrec[m] * a.n_t];
        }
      }
      for (int e = c0 + threadIdx.x + (jslow ? 0 : 256); e < c1; e += 256) {  // the uncached cells
        const int gid = a.tt.cell_gid[e];
        T acc = T(0);
        for (int q = a.tt.gcell_ptr[gid]; q < a.tt.gcell_ptr[gid + 1]; ++q)
          acc = fma_rn(a.gcell_w[q], gs[(long long)a.tt.gcell_rec[q] * a.n_t], acc);
        sjs[a.tt.cell_local[e]] = acc;
      }
    }
    __syncthreads();  // every thread's copies and cotangents of shot s are in place; shot s-1 is done
    {
      const int nb = buf == 0 ? NS - 1 : buf - 1;  // the buffer shot s-1 used
      if (s + NS - 1 < se) {
        issue(ph, gcur, sp_s + nb * PSB);
        issue(pc, gprev, sq_s + nb * QSB);
        if (grad) issue(pc, glap, sl_s + nb * QSB);
      }
      cp_async_commit();
      gcur += fs;
      gprev += fs;
      glap += fs;
    }
    const T* P = sp + buf * S::PS;
    const T* Q = sq + buf * S::QS;
    const T* LP = sl + buf * S::QS;

    T wv[2 * R + 1][VZ];  // sliding window over q^{n+1}, own columns
#pragma unroll
    for (int q = 0; q < 2 * R; ++q) vload<T, VZ>(P + (lrow + q) * S::SW + S::HL + lane * VZ, wv[q]);
#pragma unroll
    for (int k = 0; k < RX; ++k) {
      const int prow = lrow + k + R;
      vload<T, VZ>(P + (prow + R) * S::SW + S::HL + lane * VZ, wv[2 * R]);
      Row3<T, VZ> rw;
      vload<T, VZ>(P + prow * S::SW + S::HL + lane * VZ - VZ, rw.l);
#pragma unroll
      for (int v = 0; v < VZ; ++v) rw.c[v] = wv[R][v];
      vload<T, VZ>(P + prow * S::SW + S::HL + lane * VZ + VZ, rw.r);
      const int toff = (lrow + k) * S::TZ + lane * VZ;  // the owned cells in a core tile
      T q2[VZ], cc[VZ];
      vload<T, VZ>(Q + toff, q2);
      vload<T, VZ>(scc + toff, cc);
      T ca[VZ], cb[VZ], inj[VZ];
#pragma unroll
      for (int v = 0; v < VZ; ++v) { ca[v] = T(1); cb[v] = T(1); inj[v] = T(0); }
      if (layer_tile) {
        vload<T, VZ>(sa + toff, ca);
        vload<T, VZ>(sbb + toff, cb);
      }
      if (inject) vload<T, VZ>(sjs + toff, inj);
      T o[VZ];
#pragma unroll
      for (int v = 0; v < VZ; ++v) {
        const T lap = lap_at<T, R, VZ>(wv, rw, v, wc, w1x, w1z, w2x, w2z);
        o[v] = fma_rn(cc[v], inject ? add_rn(lap, inj[v]) : lap, fma_rn(-cb[v], q2[v], add_rn(wv[R][v], wv[R][v])));
      }
      if (use_a) {
#pragma unroll
        for (int v = 0; v < VZ; ++v) o[v] = mul_rn(ca[v], o[v]);
      }
      if (grad) {
        T gl[VZ];
        vload<T, VZ>(LP + toff, gl);
#pragma unroll
        for (int v = 0; v < VZ; ++v) gsum[k][v] = fma_rn(wv[R][v], gl[v], gsum[k][v]);
      }
      if (okr[k]) store_row<T, VZ>(ob + k * ld, o, zc, a.z_end);
#pragma unroll
      for (int q = 0; q < 2 * R; ++q)
#pragma unroll
        for (int v = 0; v < VZ; ++v) wv[q][v] = wv[q + 1][v];
    }
    ob += fs;
    buf = buf + 1 == NS ? 0 : buf + 1;
  }
  if (grad && own_cols) {  // the accumulator tile landed with the first commit group
    T* gp = a.gacc + (long long)bz * g.field + cbase;
#pragma unroll
    for (int k = 0; k < RX; ++k) {
      if (xr + k >= a.x_end) continue;
      T old[VZ];
      vload<T, VZ>(sg + (lrow + k) * S::TZ + lane * VZ, old);
#pragma unroll
      for (int v = 0; v < VZ; ++v) old[v] = add_rn(old[v], gsum[k][v]);
      store_row<T, VZ>(gp + (long long)k * ld, old, zc, a.z_end);
    }
  }
}

// ------------------------------------------------------------------------------------------
// Two forward steps per launch (temporal blocking): p^{n+1} and p^{n+2} of every shot of a group over
// one core tile of TX - 2R rows by TZ - 2 HL columns. The thread layout is fwd2d's over the extended
// tile E (TX x TZ: the core with R rows and HL columns around it), whose first step p^{n+1} goes to a
// shared tile; the second step reads it there, with p^n from the staged halo tile. Each cell takes
// fwd2d's arithmetic in the same order, so the fields, traces and Laplacians are bitwise those of two
// one-step launches. Cells of E outside the grid hold exact zeros in the shared p^{n+1} tile (the
// zero padding the second step's Laplacian sees); only core cells are stored. The source stencil and
// receivers of both steps are applied to the levels they belong to.
// ------------------------------------------------------------------------------------------
template <typename T, int VZ, int RX, int R>
struct Tile2T {  // the core tile of a two-step launch inside fwd2d's tile shape
  using S = Tile2Shape<T, VZ, RX, R>;
  static constexpr int CX = S::TX - 2 * R;
  static constexpr int CZ = S::TZ - 2 * S::HL;
  static constexpr int NS = (sizeof(T) == 8 || RX >= 4 || VZ >= 4) ? 2 : 3;  // shot buffers of p^n
};

template <typename T, int R, int VZ, int RX, bool AB>
__device__ __forceinline__ void fwd2t_body(const KGrid<T>& g, const Tiled2<T>& a, int bx, int by, int bz,
                                           unsigned char* smem_raw) {
  using S = Tile2Shape<T, VZ, RX, R>;
  using U = Tile2T<T, VZ, RX, R>;
  constexpr int NS = U::NS;
  T* scc = reinterpret_cast<T*>(smem_raw);  // [QS] C over E
  T* sa = scc + S::QS;                      // [QS] A (layer tiles)
  T* sbb = sa + S::QS;                      // [QS] B (layer tiles)
  T* sq = sbb + S::QS;                      // [PS] p^{n+1} over E, E at (R, HL)
  T* sp = sq + S::PS;                       // [NS][PS] p^n with halo

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cz0 = bx * U::CZ, cx0 = by * U::CX;       // core tile origin
  const int z0 = cz0 - S::HL, x0 = cx0 - R;            // E origin
  const int tile = by * a.tt.tiles_z + bx;
  const int sb = bz * a.shots_per_cta;
  const int se = min(sb + a.shots_per_cta, a.n_shots);
  const int zc = z0 + lane * VZ;  // first owned column of E
  const int xr = x0 + warp * RX;  // first owned row of E
  const int lrow = warp * RX;     // first owned row inside E
  const int ld = (int)g.s0;
  const long long cbase = g.origin + (long long)xr * ld + zc;
  const bool core_cols = lane * VZ >= S::HL && lane * VZ < S::HL + U::CZ;  // lane-uniform
  bool in_row[RX], core_row[RX];  // row k of the owned cells lies in the grid / in the core
#pragma unroll
  for (int k = 0; k < RX; ++k) {
    const int x = xr + k;
    in_row[k] = x >= 0 && x < g.n0;
    core_row[k] = lrow + k >= R && lrow + k < R + U::CX && in_row[k];
  }
  bool in_col[VZ];
#pragma unroll
  for (int v = 0; v < VZ; ++v) in_col[v] = zc + v >= 0 && zc + v < g.n1;
  const bool vec_ok = zc >= 0 && zc + VZ <= ld;  // the owned vector lies inside a row of the layout

  const bool layer_tile = AB && (x0 < g.lo0 || x0 + S::TX > g.hi0 || z0 < g.lo1 || z0 + S::TZ > g.hi1);
  const bool use_b = layer_tile && !a.b_one;  // first step: B = 1 on the first Cerjan step
  const bool use_b2 = layer_tile;             // second step (n + 1 >= 1)
  const CopyPlan<S::NCH> ph = plan_halo<T, VZ, RX, R>(g, x0, z0);
  const CopyPlan<S::NCC> pc = plan_core<T, VZ, RX, R>(g, x0, z0);
  issue(pc, a.C, smem_addr(scc));  // constants, before the wait (first commit group)
  if (layer_tile) {
    issue(pc, a.A, smem_addr(sa));
    issue(pc, a.B, smem_addr(sbb));
  }
  T pv[RX][VZ];  // p^{n-1} of the owned cells of E, one shot ahead
#pragma unroll
  for (int k = 0; k < RX; ++k) {
#pragma unroll
    for (int v = 0; v < VZ; ++v) pv[k][v] = T(0);
    if (a.prev_ready && in_row[k] && vec_ok)
      vldcg<T, VZ>(a.prev + (long long)sb * g.field + cbase + (long long)k * ld, pv[k]);
  }
  int e0 = 0, e1 = 0;
  if (a.traces || a.traces1) { e0 = a.tt.rec_ptr[tile]; e1 = a.tt.rec_ptr[tile + 1]; }
  int2 scor = make_int2(-1 << 20, -1 << 20);
  if (a.src_corner) scor = make_int2(a.src_corner[2 * sb], a.src_corner[2 * sb + 1]);
  wait_previous_grid();
  allow_next_grid();
  if (!a.prev_ready) {
#pragma unroll
    for (int k = 0; k < RX; ++k)
      if (in_row[k] && vec_ok) vldg<T, VZ>(a.prev + (long long)sb * g.field + cbase + (long long)k * ld, pv[k]);
  }
#pragma unroll
  for (int i = 0; i < NS - 1; ++i) {
    if (sb + i < se) issue(ph, a.cur + (long long)(sb + i) * g.field, smem_addr(sp + i * S::PS));
    cp_async_commit();
  }
  const T wc = g.wc, w1x = g.w1a, w1z = g.w1b, w2x = g.w2a, w2z = g.w2b;

  for (int s = sb; s < se; ++s) {
    const int buf = (s - sb) % NS;
    cp_async_wait<NS - 2>();
    __syncthreads();  // shot s landed; every thread is done with shot s-1 (its halo buffer and sq)
    {
      const int sn = s + NS - 1, nb = (sn - sb) % NS;
      if (sn < se) issue(ph, a.cur + (long long)sn * g.field, smem_addr(sp + nb * S::PS));
      cp_async_commit();
    }
    const T* P = sp + buf * S::PS;
    // receiver samples of level n (corners in the core tile; P holds E with R rows, HL columns of halo)
    if (a.traces)
      for (int e = e0 + threadIdx.x; e < e1; e += 256) {
        const int r = a.tt.rec_list[e];
        const int row = a.tt.rec_corner[2 * r] - x0 + R, col = a.tt.rec_corner[2 * r + 1] - z0 + S::HL;
        const T* w = a.rec_w + 4 * r;
        T acc = mul_rn(w[0], P[row * S::SW + col]);
        acc = fma_rn(w[1], P[row * S::SW + col + 1], acc);
        acc = fma_rn(w[2], P[(row + 1) * S::SW + col], acc);
        acc = fma_rn(w[3], P[(row + 1) * S::SW + col + 1], acc);
        a.traces[((long long)s * a.n_rec + r) * a.n_t + a.j] = acc;
      }
    const int sbx = scor.x, sbz = scor.y;
    if (a.src_corner && s + 1 < se) scor = make_int2(a.src_corner[2 * (s + 1)], a.src_corner[2 * (s + 1) + 1]);
    const bool src_tile = a.src_corner && sbx + 1 >= x0 && sbx < x0 + S::TX && sbz + 1 >= z0 && sbz < z0 + S::TZ;
    T sw0 = 0, sw1 = 0, sw2 = 0, sw3 = 0, tw0 = 0, tw1 = 0, tw2 = 0, tw3 = 0;
    if (src_tile) {
      const T wn = a.wavelet[a.n];
      sw0 = mul_rn(a.src_w[4 * s], wn); sw1 = mul_rn(a.src_w[4 * s + 1], wn);
      sw2 = mul_rn(a.src_w[4 * s + 2], wn); sw3 = mul_rn(a.src_w[4 * s + 3], wn);
      if (a.two) {
        const T wm = a.wavelet[a.n + 1];
        tw0 = mul_rn(a.src_w[4 * s], wm); tw1 = mul_rn(a.src_w[4 * s + 1], wm);
        tw2 = mul_rn(a.src_w[4 * s + 2], wm); tw3 = mul_rn(a.src_w[4 * s + 3], wm);
      }
    }
    const bool more = s + 1 < se;
    const long long so = (long long)s * g.field, sn = so + g.field;

    // ---- step n over E: p^{n+1} into sq (zeros outside the grid), core cells to global
    {
      T wv[2 * R + 1][VZ];
#pragma unroll
      for (int q = 0; q < 2 * R; ++q) vload<T, VZ>(P + (lrow + q) * S::SW + S::HL + lane * VZ, wv[q]);
#pragma unroll
      for (int k = 0; k < RX; ++k) {
        const int prow = lrow + k + R;
        vload<T, VZ>(P + (prow + R) * S::SW + S::HL + lane * VZ, wv[2 * R]);
        Row3<T, VZ> rw;
        vload<T, VZ>(P + prow * S::SW + S::HL + lane * VZ - VZ, rw.l);
#pragma unroll
        for (int v = 0; v < VZ; ++v) rw.c[v] = wv[R][v];
        vload<T, VZ>(P + prow * S::SW + S::HL + lane * VZ + VZ, rw.r);
        const int x = xr + k;
        const int toff = (lrow + k) * S::TZ + lane * VZ;
        T cc[VZ], ca[VZ], cb[VZ];
        vload<T, VZ>(scc + toff, cc);
#pragma unroll
        for (int v = 0; v < VZ; ++v) { ca[v] = T(1); cb[v] = T(1); }
        if (layer_tile) vload<T, VZ>(sa + toff, ca);
        if (use_b) vload<T, VZ>(sbb + toff, cb);
        T o[VZ], lp[VZ];
#pragma unroll
        for (int v = 0; v < VZ; ++v) {
          lp[v] = lap_at<T, R, VZ>(wv, rw, v, wc, w1x, w1z, w2x, w2z);
          o[v] = fma_rn(cc[v], lp[v], fma_rn(-cb[v], pv[k][v], add_rn(wv[R][v], wv[R][v])));
        }
        if (src_tile) {
#pragma unroll
          for (int v = 0; v < VZ; ++v) {
            const int dx = x - sbx, dz = zc + v - sbz;
            if (dx >= 0 && dx <= 1 && dz >= 0 && dz <= 1)
              o[v] = add_rn(o[v], (dx == 0) ? (dz == 0 ? sw0 : sw1) : (dz == 0 ? sw2 : sw3));
          }
        }
        if (layer_tile) {
#pragma unroll
          for (int v = 0; v < VZ; ++v) o[v] = mul_rn(ca[v], o[v]);
        }
        if (core_row[k] && core_cols) {
          const long long ro = cbase + (long long)k * ld;
          store_row<T, VZ>(a.next + so + ro, o, zc, g.n1);
          if (a.lap_out) store_row<T, VZ>(a.lap_out + so + ro, lp, zc, g.n1);
        }
        if (a.two) {
#pragma unroll
          for (int v = 0; v < VZ; ++v)
            if (!(in_row[k] && in_col[v])) o[v] = T(0);  // the grid's zero padding for the next step
          vstore<T, VZ>(sq + prow * S::SW + S::HL + lane * VZ, o);
        }
        if (more && in_row[k] && vec_ok) vldg<T, VZ>(a.prev + sn + cbase + (long long)k * ld, pv[k]);
#pragma unroll
        for (int q = 0; q < 2 * R; ++q)
#pragma unroll
          for (int v = 0; v < VZ; ++v) wv[q][v] = wv[q + 1][v];
      }
    }
    if (!a.two) continue;
    __syncthreads();  // p^{n+1} of all of E is in sq
    if (a.traces1)  // receiver samples of level n+1
      for (int e = e0 + threadIdx.x; e < e1; e += 256) {
        const int r = a.tt.rec_list[e];
        const int row = a.tt.rec_corner[2 * r] - x0 + R, col = a.tt.rec_corner[2 * r + 1] - z0 + S::HL;
        const T* w = a.rec_w + 4 * r;
        T acc = mul_rn(w[0], sq[row * S::SW + col]);
        acc = fma_rn(w[1], sq[row * S::SW + col + 1], acc);
        acc = fma_rn(w[2], sq[(row + 1) * S::SW + col], acc);
        acc = fma_rn(w[3], sq[(row + 1) * S::SW + col + 1], acc);
        a.traces1[((long long)s * a.n_rec + r) * a.n_t + a.j1] = acc;
      }
    // ---- step n+1 over E (kept only in the core): p^{n+2} from sq, p^n from the halo tile's centre
    {
      T wv[2 * R + 1][VZ];
#pragma unroll
      for (int q = 0; q < 2 * R; ++q) vload<T, VZ>(sq + (lrow + q) * S::SW + S::HL + lane * VZ, wv[q]);
#pragma unroll
      for (int k = 0; k < RX; ++k) {
        const int prow = lrow + k + R;
        vload<T, VZ>(sq + (prow + R) * S::SW + S::HL + lane * VZ, wv[2 * R]);
        Row3<T, VZ> rw;
        vload<T, VZ>(sq + prow * S::SW + S::HL + lane * VZ - VZ, rw.l);
#pragma unroll
        for (int v = 0; v < VZ; ++v) rw.c[v] = wv[R][v];
        vload<T, VZ>(sq + prow * S::SW + S::HL + lane * VZ + VZ, rw.r);
        const int x = xr + k;
        const int toff = (lrow + k) * S::TZ + lane * VZ;
        T cc[VZ], ca[VZ], cb[VZ], pn[VZ];
        vload<T, VZ>(scc + toff, cc);
        vload<T, VZ>(P + prow * S::SW + S::HL + lane * VZ, pn);  // p^n at the owned cells
#pragma unroll
        for (int v = 0; v < VZ; ++v) { ca[v] = T(1); cb[v] = T(1); }
        if (layer_tile) vload<T, VZ>(sa + toff, ca);
        if (use_b2) vload<T, VZ>(sbb + toff, cb);
        T o[VZ], lp[VZ];
#pragma unroll
        for (int v = 0; v < VZ; ++v) {
          lp[v] = lap_at<T, R, VZ>(wv, rw, v, wc, w1x, w1z, w2x, w2z);
          o[v] = fma_rn(cc[v], lp[v], fma_rn(-cb[v], pn[v], add_rn(wv[R][v], wv[R][v])));
        }
        if (src_tile) {
#pragma unroll
          for (int v = 0; v < VZ; ++v) {
            const int dx = x - sbx, dz = zc + v - sbz;
            if (dx >= 0 && dx <= 1 && dz >= 0 && dz <= 1)
              o[v] = add_rn(o[v], (dx == 0) ? (dz == 0 ? tw0 : tw1) : (dz == 0 ? tw2 : tw3));
          }
        }
        if (layer_tile) {
#pragma unroll
          for (int v = 0; v < VZ; ++v) o[v] = mul_rn(ca[v], o[v]);
        }
        if (core_row[k] && core_cols) {
          const long long ro = cbase + (long long)k * ld;
          store_row<T, VZ>(a.next2 + so + ro, o, zc, g.n1);
          if (a.lap_out1) store_row<T, VZ>(a.lap_out1 + so + ro, lp, zc, g.n1);
        }
#pragma unroll
        for (int q = 0; q < 2 * R; ++q)
#pragma unroll
          for (int v = 0; v < VZ; ++v) wv[q][v] = wv[q + 1][v];
      }
    }
  }
}

template <typename T, int R, int VZ, int RX, bool AB>
__global__ void __launch_bounds__(256, 2) fwd2t(KGrid<T> g, Tiled2<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  fwd2t_body<T, R, VZ, RX, AB>(g, a, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// The per-CTA launches of one problem: blockIdx = (tile along z, tile along x, shot group).
template <typename T, int R, int VZ, int RX, bool AB>
__global__ void __launch_bounds__(256, 4) fwd2d(KGrid<T> g, Tiled2<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  fwd2d_body<T, R, VZ, RX, AB>(g, a, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}
template <typename T, int R, int VZ, int RX, bool AB>
__global__ void __launch_bounds__(256, 3) adj2d(KGrid<T> g, Tiled2<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  adj2d_body<T, R, VZ, RX, AB>(g, a, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// ------------------------------------------------------------------------------------------
// Batched steps: one launch advances every active problem of a batch (grids of different size,
// shot counts and step counts) by one step. All problems share the global step index n (the
// forward runs n upwards from 0, the adjoint downwards from the largest step count, so a problem
// with N steps takes part in forward steps n < N and adjoint steps n <= N); the host sorts the
// problems by step count, so the active ones are a prefix of the table and the launch covers
// cta_start[n_active] CTAs. CTA b finds its problem by binary search over cta_start, builds that
// problem's step descriptor in shared memory and runs the same body as the one-problem kernels.
// ------------------------------------------------------------------------------------------
template <typename T>
struct BatchProb {
  KGrid<T> g;
  Tiled2<T> fwd, adj;  // the step-independent fields of the forward and adjoint descriptors
  T* ring;             // 3 levels of p
  T* work;             // 3 levels of q
  T* segbuf;           // `segment` levels of Lap p, level n % segment
  T* traces;
  long long level;     // elements of one level: n_shots * field
  int n_steps, substeps, first_b_one;
  int ftx, atx;        // tiles along x of the forward and adjoint tile shapes
};

__device__ __forceinline__ int batch_problem(const int* __restrict__ cta_start, int n_active, int b) {
  int lo = 0, hi = n_active - 1;  // last problem whose first CTA is <= b
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cta_start[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// store_lap != 0: a recompute step that stores Lap p^n into the segment buffer and records no
// traces; otherwise a forward-sweep step that records traces on the problem's record steps.
template <typename T, int R, int VZ, int RX>
__global__ void __launch_bounds__(256, 4) fwd2d_batch(const BatchProb<T>* __restrict__ probs,
                                                      const int* __restrict__ cta_start, int n_active, int n,
                                                      int store_lap, int segment) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ KGrid<T> sg;
  __shared__ Tiled2<T> st;
  __shared__ int sidx[3];
  if (threadIdx.x == 0) {  // the tables are written once, before any step: read before the wait
    const int p = batch_problem(cta_start, n_active, blockIdx.x);
    const BatchProb<T>& P = probs[p];
    int local = blockIdx.x - cta_start[p];
    const int tz = P.fwd.tt.tiles_z;
    sidx[0] = local % tz;
    local /= tz;
    sidx[1] = local % P.ftx;
    sidx[2] = local / P.ftx;
    sg = P.g;
    Tiled2<T> t = P.fwd;
    t.prev = P.ring + (long long)(n % 3) * P.level;
    t.cur = P.ring + (long long)((n + 1) % 3) * P.level;
    t.next = P.ring + (long long)((n + 2) % 3) * P.level;
    t.b_one = (n == 0 && P.first_b_one) ? 1 : 0;
    // a recompute segment starts from decoded snapshots, the sweep from the initial state: the
    // launch just before wrote p^{n-1}
    t.prev_ready = store_lap ? (n % segment != 0) : (n > 0);
    t.n = n;
    t.traces = (!store_lap && P.traces && t.n_rec > 0 && n % P.substeps == 0) ? P.traces : nullptr;
    t.j = n / P.substeps;
    t.lap_out = store_lap ? P.segbuf + (long long)(n % segment) * P.level : nullptr;
    st = t;
  }
  __syncthreads();
  fwd2d_body<T, R, VZ, RX, true>(sg, st, sidx[0], sidx[1], sidx[2], smem_raw);
}

template <typename T, int R, int VZ, int RX>
__global__ void __launch_bounds__(256, 3) adj2d_batch(const BatchProb<T>* __restrict__ probs,
                                                      const int* __restrict__ cta_start, int n_active, int n,
                                                      int segment) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ KGrid<T> sg;
  __shared__ Tiled2<T> st;
  __shared__ int sidx[3];
  if (threadIdx.x == 0) {
    const int p = batch_problem(cta_start, n_active, blockIdx.x);
    const BatchProb<T>& P = probs[p];
    int local = blockIdx.x - cta_start[p];
    const int tz = P.adj.tt.tiles_z;
    sidx[0] = local % tz;
    local /= tz;
    sidx[1] = local % P.atx;
    sidx[2] = local / P.atx;
    sg = P.g;
    Tiled2<T> t = P.adj;
    t.cur = P.work + (long long)((n + 1) % 3) * P.level;
    t.prev = P.work + (long long)((n + 2) % 3) * P.level;
    t.next = P.work + (long long)(n % 3) * P.level;
    t.apply_a = n >= 1 ? 1 : 0;
    t.lap = n < P.n_steps ? P.segbuf + (long long)(n % segment) * P.level : nullptr;
    // the first adjoint step of a segment directly follows the recompute step that wrote its Lap p
    // (a segment ends at a multiple of `segment` or at the batch's last step, problem 0's step count)
    t.lap_ready = (n + 1) % segment != 0 && n + 1 != probs[0].n_steps;
    if (n % P.substeps != 0) t.gtr = nullptr;  // the descriptor holds the cotangents
    t.j = n / P.substeps;
    st = t;
  }
  __syncthreads();
  adj2d_body<T, R, VZ, RX, true>(sg, st, sidx[0], sidx[1], sidx[2], smem_raw);
}

}  // namespace nw
