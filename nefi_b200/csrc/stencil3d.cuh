// stencil3d.cuh — plane-marching 3-D leapfrog step for sm_100a (forward and q-form adjoint).
//
// A CTA (8 warps) owns a (y, z) tile of TY = 8 rows by TZ = 32*VZ columns and marches along x over
// a chunk of XC planes. Warp w owns row y0 + w, lane l the VZ columns z0 + l*VZ. Every plane the
// march touches passes once through a ring of NSP shared-memory tiles, (TY + 2R) rows by
// TZ + 2*HL columns (the y/z halo), staged by cp.async two planes ahead of its first use (one
// barrier per plane: a plane's copy is issued right after the barrier that frees its slot); the
// x-neighbours of a thread's cells stay in a (2R+1)-plane register window, fed from the ring when a
// plane arrives. The y/z neighbours of the centre plane come from its shared tile. Planes outside
// the grid are never copied: their window values are zero, like the ghost planes they stand for.
// C, p^{n-1} (q^{n+2}), the stored Lap p and the gradient accumulator are read at the thread's own
// cells straight from global memory with vector loads issued one plane ahead; A/B (layer cells) when
// needed.
#pragma once
#include "kernels.cuh"
#include "stencil2d.cuh"

namespace nw {

template <typename T, int VZ, int R>
struct Tile3Shape {
  static constexpr int NT = 256;                 // threads per CTA: one warp per tile row
  static constexpr int TY = NT / 32;
  static constexpr int TZ = 32 * VZ;
  static constexpr int HL = 16 / (int)sizeof(T);
  static constexpr int SW = TZ + 2 * HL;
  static constexpr int EPC = 16 / (int)sizeof(T);
  static constexpr int HR = TY + 2 * R;
  static constexpr int PS = HR * SW;                        // elements of a plane tile
  static constexpr int NCH = (HR * (SW / EPC) + NT - 1) / NT;  // chunks per thread and plane
  static constexpr int NSP = R + 3;                          // planes in the ring
};

// The chunks of one plane tile: element offsets from the field base for plane 0 (add x * s0 for
// plane x; they are >= 0 for x >= 0 thanks to the ghost planes and the guard, and -1 marks a chunk
// that is not copied); rows and columns that no output cell reads (beyond the ghost rows, past the
// row pitch) are not copied.
template <typename T, int VZ, int R>
__device__ __forceinline__ CopyPlan<Tile3Shape<T, VZ, R>::NCH> plan_plane(const KGrid<T>& g, int y0, int z0) {
  using S = Tile3Shape<T, VZ, R>;
  constexpr int CPR = S::SW / S::EPC;
  CopyPlan<S::NCH> p;
#pragma unroll
  for (int i = 0; i < S::NCH; ++i) {
    const int c = threadIdx.x + S::NT * i;
    const int row = c / CPR, ch = c - row * CPR;
    const int y = y0 - R + row;
    const int z = z0 - S::HL + ch * S::EPC;
    p.soff[i] = (unsigned)((row * S::SW + ch * S::EPC) * sizeof(T));
    p.goff[i] = (c < S::HR * CPR && y < g.n1 + R && z < (int)g.s1) ? (int)(g.origin + (long long)y * g.s1 + z) : -1;
  }
  return p;
}

template <typename T, int R, int VZ, bool ADJ>
__global__ void __launch_bounds__(Tile3Shape<T, VZ, R>::NT, sizeof(T) == 8 ? 3 : 4) step3t(KGrid<T> g, Step3<T> a, int xc, int n_shots) {
  using S = Tile3Shape<T, VZ, R>;
  constexpr int NSP = S::NSP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);  // [NSP][PS]
  const unsigned ring_sa = smem_addr(ring);

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // grid.x = tile * n_shots + shot (the shot fastest, so that the CTAs of one tile for all shots run
  // together and the shot-independent fields C, A, B come from L2 after the first), grid.y = x chunk
  const int tiles_z = (g.n2 + S::TZ - 1) / S::TZ;
  const int s = blockIdx.x % n_shots, tile = blockIdx.x / n_shots;
  const int z0 = (tile % tiles_z) * S::TZ, y0 = (tile / tiles_z) * S::TY;
  const int x0 = blockIdx.y * xc, x1 = min(x0 + xc, g.n0);
  const long long so = (long long)s * g.field;
  const int y = y0 + warp, zc = z0 + lane * VZ;
  const bool own = y < g.n1 && zc < g.n2;
  const long long ld = g.s1;
  const T* __restrict__ cur = a.cur + so;
  const CopyPlan<S::NCH> pp = plan_plane<T, VZ, R>(g, y0, z0);
  // the planes of the march: xa = x0 - R .. xb - 1 = x1 + R - 1; plane p sits in ring slot
  // (p - xa) % NSP. When plane p is consumed (its own cells enter the window front) the centre is
  // p - R: planes p - R .. p must be resident, and the copy of plane p + 2 goes into the slot of
  // plane p - R - 1 (NSP = R + 3), the centre of the previous iteration.
  const int xa = x0 - R, xb = x1 + R;
  auto issue_plane = [&](int p) {
    if (p >= 0 && p < g.n0 && p < xb) issue(pp, cur + (long long)p * g.s0, ring_sa + ((p - xa) % NSP) * (unsigned)(S::PS * sizeof(T)));
  };
  wait_previous_grid();
  allow_next_grid();
  if (!ADJ && a.traces)
    gather_receivers<T, 8>(cur, a.traces, a.rec_idx, a.rec_w, a.n_rec, a.n_t, a.j, s,
                           ((long long)blockIdx.y * (gridDim.x / n_shots) + tile) * blockDim.x + threadIdx.x,
                           (long long)(gridDim.x / n_shots) * gridDim.y * blockDim.x);
  issue_plane(xa);  // one commit group per plane, empty groups included
  cp_async_commit();
  issue_plane(xa + 1);
  cp_async_commit();
  const bool yz_layer = y0 < g.lo1 || y0 + S::TY > g.hi1 || z0 < g.lo2 || z0 + S::TZ > g.hi2;
  const T wc = g.wc, w1x = g.w1a, w1y = g.w1b, w1z = g.w1c, w2x = g.w2a, w2y = g.w2b, w2z = g.w2c;
  // source corners of this shot (forward)
  int bx = -4, by = -4, bz = -4;
  if (!ADJ && a.src_corner) { bx = a.src_corner[3 * s]; by = a.src_corner[3 * s + 1]; bz = a.src_corner[3 * s + 2]; }

  T wv[2 * R + 1][VZ];  // own cells of planes p - 2R .. p
#pragma unroll
  for (int q = 0; q < 2 * R + 1; ++q)
#pragma unroll
    for (int v = 0; v < VZ; ++v) wv[q][v] = T(0);
  const int own_off = (warp + R) * S::SW + S::HL + lane * VZ;
  // the per-cell fields of the next plane's own cells, loaded one plane ahead into registers
  const long long row_off = g.origin + (long long)y * ld + zc;  // + x * s0
  T pvn[VZ], ccn[VZ], gln[VZ], ggn[VZ];
  auto prefetch = [&](int x) {
    if (x < x1 && own) {
      const long long i = row_off + (long long)x * g.s0;
      vldg<T, VZ>(a.prev + so + i, pvn);
      vldg<T, VZ>(a.C + i, ccn);
      if (ADJ && a.lap) {
        vldg<T, VZ>(a.lap + so + i, gln);
        vload<T, VZ>(a.grad + so + i, ggn);
      }
    }
  };
  prefetch(x0);
  for (int p = xa; p < xb; ++p) {
    cp_async_wait<1>();  // this thread's copies of plane p have landed
    __syncthreads();     // everyone's have, and every thread is done with the previous centre's slot
    issue_plane(p + 2);  // into that slot
    cp_async_commit();
    if (p >= 0 && p < g.n0) vload<T, VZ>(ring + ((p - xa) % NSP) * S::PS + own_off, wv[2 * R]);
    else {
#pragma unroll
      for (int v = 0; v < VZ; ++v) wv[2 * R][v] = T(0);
    }
    const int x = p - R;
    if (x >= x0 && own) {
      const T* P = ring + ((x - xa) % NSP) * S::PS;  // the centre plane's tile
      const long long i = g.origin + (long long)x * g.s0 + (long long)y * ld + zc;
      Row3<T, VZ> rw;
      vload<T, VZ>(P + own_off - VZ, rw.l);
#pragma unroll
      for (int v = 0; v < VZ; ++v) rw.c[v] = wv[R][v];
      vload<T, VZ>(P + own_off + VZ, rw.r);
      T ym[VZ], yp[VZ], ym2[VZ], yp2[VZ];
      vload<T, VZ>(P + own_off - S::SW, ym);
      vload<T, VZ>(P + own_off + S::SW, yp);
      if (R == 2) {
        vload<T, VZ>(P + own_off - 2 * S::SW, ym2);
        vload<T, VZ>(P + own_off + 2 * S::SW, yp2);
      }
      T pv[VZ], cc[VZ], ca[VZ], cb[VZ], gl[VZ], gg[VZ];
#pragma unroll
      for (int v = 0; v < VZ; ++v) {
        pv[v] = pvn[v];
        cc[v] = ccn[v];
        gl[v] = gln[v];
        gg[v] = ggn[v];
      }
      prefetch(x + 1);  // in flight while this plane is computed
      const bool layer = yz_layer || x < g.lo0 || x >= g.hi0;
#pragma unroll
      for (int v = 0; v < VZ; ++v) { ca[v] = T(1); cb[v] = T(1); }
      if (a.A && layer) {
        vldg<T, VZ>(a.A + i, ca);
        if (ADJ || !a.b_one) vldg<T, VZ>(a.B + i, cb);
      }
      T o[VZ], lp[VZ];
#pragma unroll
      for (int v = 0; v < VZ; ++v) {
        const T c = wv[R][v];
        T lap = fma_rn(w1z, add_rn(zval(rw, v - 1), zval(rw, v + 1)),
                       fma_rn(w1y, add_rn(ym[v], yp[v]),
                              fma_rn(w1x, add_rn(wv[R - 1][v], wv[R + 1][v]), mul_rn(wc, c))));
        if (R == 2)
          lap = fma_rn(w2z, add_rn(zval(rw, v - 2), zval(rw, v + 2)),
                       fma_rn(w2y, add_rn(ym2[v], yp2[v]), fma_rn(w2x, add_rn(wv[0][v], wv[4][v]), lap)));
        lp[v] = lap;
        o[v] = fma_rn(cc[v], lap, fma_rn(-cb[v], pv[v], add_rn(c, c)));
      }
      if (!ADJ && bx >= x - 1 && bx <= x && by >= y - 1 && by <= y) {  // the source stencil touches this row
        const T wn = a.wavelet[a.n];
#pragma unroll
        for (int v = 0; v < VZ; ++v) {
          const int dx = x - bx, dy = y - by, dz = zc + v - bz;
          if (dz >= 0 && dz <= 1) o[v] = add_rn(o[v], mul_rn(a.src_w[8 * s + 4 * dx + 2 * dy + dz], wn));
        }
      }
      if (layer && a.A && (!ADJ || a.apply_a)) {
#pragma unroll
        for (int v = 0; v < VZ; ++v) o[v] = mul_rn(ca[v], o[v]);
      }
      store_row<T, VZ>(a.next + so + i, o, zc, g.n2);
      if (!ADJ && a.lap_out) store_row<T, VZ>(a.lap_out + so + i, lp, zc, g.n2);
      if (ADJ && a.lap) {
#pragma unroll
        for (int v = 0; v < VZ; ++v) gg[v] = fma_rn(wv[R][v], gl[v], gg[v]);
        store_row<T, VZ>(a.grad + so + i, gg, zc, g.n2);
      }
    }
#pragma unroll
    for (int q = 0; q < 2 * R; ++q)
#pragma unroll
      for (int v = 0; v < VZ; ++v) wv[q][v] = wv[q + 1][v];
  }
}

}  // namespace nw
