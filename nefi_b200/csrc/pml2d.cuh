// pml2d.cuh — 2-D leapfrog steps with the reference's PML (nefi/physics/wave.py:476-501, 529-552).
//
// Forward step k, with face differences D+ (zero outside the grid) and cell differences D- of
// face arrays, per axis ax:
//   psi_k = alpha psi_{k-1} + beta D+ p^k                                        (faces)
//   L_k   = Lap p^k + sum_ax (0.5/h_ax) D-(psi_k + psi_{k-1})
//   p^{k+1} = A (2 p^k - B p^{k-1} + C L_k - ZZ p^k + S w(k))
// Adjoint, advancing q = C mu like the other adjoint steps (D+^T = -D-, D-^T = -D+):
//   Psi_k = alpha Psi_{k+1} - (0.5/h) D+(q^{k+1} + q^{k+2})                       (faces)
//   q^k   = A (2 q^{k+1} - ZZ q^{k+1} - B q^{k+2} + C (Lap q^{k+1} - sum_ax D-(beta Psi_k)))
// and C dJ/dC += q^{k+1} L_k with L_k stored by the forward step. The receiver cotangents are
// added by inject_kernel after the step, like the 3-D adjoint.
//
// Face f of axis ax (between cells f-1 and f, f = 0..P_ax) is stored at the cell index of f in the
// ghost layout: face P_ax lands in the first ghost row (x) or column (z), which the layout always
// has. Thread (x, z) computes its own face and the next one (f = x, x+1), writes its own, and the
// last cell of a row or column also writes face P_ax. psi and Psi are double buffered by step
// parity, so no thread reads a face another thread of the same step writes.
#pragma once
#include "kernels.cuh"
#include "stencil2d.cuh"

namespace nw {

template <typename T>
struct PmlStep {
  const T* __restrict__ prev;   // forward p^{k-1} | adjoint q^{k+2}
  const T* __restrict__ cur;    // forward p^k     | adjoint q^{k+1}
  T* __restrict__ next;         // forward p^{k+1} | adjoint q^k
  const T* __restrict__ C;
  const T* __restrict__ A;
  const T* __restrict__ B;
  const T* __restrict__ ZZ;
  const T* __restrict__ alpha[2];
  const T* __restrict__ beta[2];
  const T* __restrict__ f_old[2];  // psi_{k-1} | Psi_{k+1} (per shot at +field)
  T* __restrict__ f_new[2];        // psi_k     | Psi_k
  T hx2, hz2;                      // 0.5 / h per axis
  int cx0, cx1, cz0, cz1;          // core box: every PML term vanishes exactly, the faces are skipped
  int kx0, kx1, kz0, kz1;          // a box inside the core box that a tiled kernel steps instead:
                                   // this kernel enumerates only the cells outside it (all 0: none)
  int apply_a;                     // adjoint: A applies (k >= 1)
  // forward: point sources and the stored Laplacian
  const int* __restrict__ src_corner;
  const T* __restrict__ src_w;
  const T* __restrict__ wavelet;
  int n;
  T* __restrict__ lap_out;
  // adjoint: the gradient
  const T* __restrict__ lap;
  T* __restrict__ grad;            // per-shot accumulators of C dJ/dC
};

template <typename T, int R, bool ADJ>
__global__ void __launch_bounds__(256) pml2d_step(KGrid<T> g, PmlStep<T> a) {
  wait_previous_grid();
  allow_next_grid();
  const int s = blockIdx.y;
  const long long so = (long long)s * g.field;
  // thread t -> the t-th cell outside the tiled box, row by row: the rows above it, the left and right
  // strips beside it, the rows below it (32-bit arithmetic: a field holds fewer than 2^31 cells)
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int top = a.kx0 * g.n1;
  const int bw = a.kz0 + (g.n1 - a.kz1);
  const int mid = (a.kx1 - a.kx0) * bw;
  if (t >= top + mid + (g.n0 - a.kx1) * g.n1) return;
  int x, z;
  if (t < top) {
    x = t / g.n1;
    z = t - x * g.n1;
  } else if (t < top + mid) {
    const int u = t - top;
    const int q = u / bw;
    const int r = u - q * bw;
    x = a.kx0 + q;
    z = r < a.kz0 ? r : a.kz1 + (r - a.kz0);
  } else {
    const int u = t - top - mid;
    x = a.kx1 + u / g.n1;
    z = u - (x - a.kx1) * g.n1;
  }
  const long long ld = g.s0;
  const long long i = g.origin + x * ld + z;
  const T* __restrict__ pc = a.cur + so;
  const T* __restrict__ pp = a.prev + so;
  const T c = pc[i];
  // 5- or 9-point Laplacian in the reference's zero-padded convolution (fixed rounding sequence)
  T lap = fma_rn(g.w1b, add_rn(pc[i - 1], pc[i + 1]), fma_rn(g.w1a, add_rn(pc[i - ld], pc[i + ld]), mul_rn(g.wc, c)));
  if (R == 2)
    lap = fma_rn(g.w2b, add_rn(pc[i - 2], pc[i + 2]), fma_rn(g.w2a, add_rn(pc[i - 2 * ld], pc[i + 2 * ld]), lap));
  // the faces f = x, x+1 (axis 0, stride ld) and f = z, z+1 (axis 1, stride 1)
  T pml = T(0);    // forward: sum_ax (0.5/h) D-(psi_k + psi_{k-1});  adjoint: sum_ax D-(beta Psi_k)
  // Inside the core box the faces contribute exact zeros (forward: psi stays zero there, alpha = 1,
  // beta = 0; adjoint: beta = 0 multiplies the face cotangents) and A = B = 1, ZZ = 0, so the cell
  // takes the same rounding sequence with those constants and neither reads nor writes a face.
  const bool core = x >= a.cx0 && x < a.cx1 && z >= a.cz0 && z < a.cz1;
#pragma unroll
  for (int ax = 0; ax < 2; ++ax) {
    if (core) break;
    const long long st = ax == 0 ? ld : 1;
    const long long j = i + st;  // index of face f+1
    const T* __restrict__ al = a.alpha[ax];
    const T* __restrict__ be = a.beta[ax];
    const T* __restrict__ fo = a.f_old[ax] + so;
    T f0, f1;
    if (!ADJ) {  // psi_k = alpha psi_{k-1} + beta (p[f] - p[f-1])
      f0 = fma_rn(be[i], add_rn(c, -pc[i - st]), mul_rn(al[i], fo[i]));
      f1 = fma_rn(be[j], add_rn(pc[j], -c), mul_rn(al[j], fo[j]));
      const T h2 = ax == 0 ? a.hx2 : a.hz2;
      pml = fma_rn(h2, add_rn(add_rn(f1, fo[j]), -add_rn(f0, fo[i])), pml);
    } else {  // Psi_k = alpha Psi_{k+1} - (0.5/h)(s[f] - s[f-1]),  s = q^{k+1} + q^{k+2}
      const T h2 = ax == 0 ? a.hx2 : a.hz2;
      const T sm = add_rn(pc[i - st], pp[i - st]), s0 = add_rn(c, pp[i]), sp = add_rn(pc[j], pp[j]);
      f0 = fma_rn(-h2, add_rn(s0, -sm), mul_rn(al[i], fo[i]));
      f1 = fma_rn(-h2, add_rn(sp, -s0), mul_rn(al[j], fo[j]));
      pml = add_rn(pml, add_rn(mul_rn(be[j], f1), -mul_rn(be[i], f0)));
    }
    T* __restrict__ fn = a.f_new[ax] + so;
    fn[i] = f0;
    if ((ax == 0 ? x : z) == (ax == 0 ? g.n0 : g.n1) - 1) fn[j] = f1;  // the last face of the axis
  }
  const T av = core ? T(1) : a.A[i], bv = core ? T(1) : a.B[i], zz = core ? T(0) : a.ZZ[i], cc = a.C[i];
  T o;
  if (!ADJ) {
    const T L = add_rn(lap, pml);
    if (a.lap_out) a.lap_out[so + i] = L;
    o = fma_rn(-zz, c, fma_rn(cc, L, fma_rn(-bv, pp[i], add_rn(c, c))));
    if (a.src_corner) {
      const int bx = a.src_corner[2 * s], bz = a.src_corner[2 * s + 1];
      const int dx = x - bx, dz = z - bz;
      if (dx >= 0 && dx <= 1 && dz >= 0 && dz <= 1) o = add_rn(o, mul_rn(a.src_w[4 * s + 2 * dx + dz], a.wavelet[a.n]));
    }
    a.next[so + i] = mul_rn(av, o);
  } else {
    o = fma_rn(-bv, pp[i], fma_rn(cc, add_rn(lap, -pml), fma_rn(-zz, c, add_rn(c, c))));
    a.next[so + i] = a.apply_a ? mul_rn(av, o) : o;
    if (a.lap) a.grad[so + i] = fma_rn(c, a.lap[so + i], a.grad[so + i]);
  }
}

// ------------------------------------------------------------------------------------------
// The layer cells outside a tiled interior box [kx0, kx1) x [kz0, kz1), in chunks of CW = 16 bytes /
// sizeof(T) consecutive cells of a row (kz0 is chunk-aligned; a chunk may reach into the box past
// kz1 or past the last column, and such cells are neither written nor their faces): thread t owns
// layer chunk t of the rows above the box, the strips left and right of it, and the rows below it,
// in that order. A CTA loops over a group of shots, the cells' coefficients (C, A, B, ZZ and the face
// coefficients of both axes) staying in registers across the group; every field access is a
// coalesced 16-byte vector load or store. Each cell takes exactly the arithmetic of pml2d_step, so
// the two kernels give bitwise the same fields.
// ------------------------------------------------------------------------------------------
template <typename T>
struct PmlChunks {
  int nch;                  // chunks per row (ceil(n1 / CW))
  int ka, kb;               // chunks of a middle row left of the box: [0, ka); right of it: [kb, nch)
  int n_top, n_mid, n_all;  // chunks in the rows above the box, in the middle rows, in all
  int spc;                  // shots per CTA
};

template <typename T>
__host__ __device__ inline PmlChunks<T> pml_chunks(int n0, int n1, int kx0, int kx1, int kz0, int kz1, int spc) {
  constexpr int CW = 16 / (int)sizeof(T);
  PmlChunks<T> c;
  c.nch = (n1 + CW - 1) / CW;
  c.ka = kz0 / CW;
  c.kb = kz1 / CW;
  c.n_top = kx0 * c.nch;
  c.n_mid = (kx1 - kx0) * (c.ka + c.nch - c.kb);
  c.n_all = c.n_top + c.n_mid + (n0 - kx1) * c.nch;
  c.spc = spc;
  return c;
}

template <typename T, int R, bool ADJ>
__global__ void __launch_bounds__(128) pml2d_chunk_step(KGrid<T> g, PmlStep<T> a, PmlChunks<T> ck, int n_shots) {
  constexpr int CW = 16 / (int)sizeof(T);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = t < ck.n_all;
  int x = 0, zc = 0;
  if (t < ck.n_top) {
    x = t / ck.nch;
    zc = (t - x * ck.nch) * CW;
  } else if (t < ck.n_top + ck.n_mid) {
    const int u = t - ck.n_top, w = ck.ka + ck.nch - ck.kb;
    const int q = u / w, r = u - q * w;
    x = a.kx0 + q;
    zc = (r < ck.ka ? r : ck.kb + (r - ck.ka)) * CW;
  } else if (live) {
    const int u = t - ck.n_top - ck.n_mid;
    x = a.kx1 + u / ck.nch;
    zc = (u - (x - a.kx1) * ck.nch) * CW;
  }
  const long long ld = g.s0;
  const long long i = g.origin + x * ld + zc;
  // which cells of the chunk are layer cells of the grid, and which lie in the core box
  bool own[CW], core[CW];
  bool all_own = live;
#pragma unroll
  for (int v = 0; v < CW; ++v) {
    const int z = zc + v;
    own[v] = live && z < g.n1 && (x < a.kx0 || x >= a.kx1 || z < a.kz0 || z >= a.kz1);
    core[v] = x >= a.cx0 && x < a.cx1 && z >= a.cz0 && z < a.cz1;
    all_own = all_own && own[v];
  }
  // shot-independent coefficients, loaded before the wait (constant over the sweep)
  T C[CW], A[CW], B[CW], ZZ[CW], al0[CW], al0n[CW], be0[CW], be0n[CW], al1[CW + 1], be1[CW + 1];
  if (live) {
    vldcg<T, CW>(a.C + i, C);
    vldcg<T, CW>(a.A + i, A);
    vldcg<T, CW>(a.B + i, B);
    vldcg<T, CW>(a.ZZ + i, ZZ);
    vldcg<T, CW>(a.alpha[0] + i, al0);
    vldcg<T, CW>(a.alpha[0] + i + ld, al0n);
    vldcg<T, CW>(a.beta[0] + i, be0);
    vldcg<T, CW>(a.beta[0] + i + ld, be0n);
    T tmp[CW];
    vldcg<T, CW>(a.alpha[1] + i, tmp);
#pragma unroll
    for (int v = 0; v < CW; ++v) al1[v] = tmp[v];
    al1[CW] = a.alpha[1][i + CW];
    vldcg<T, CW>(a.beta[1] + i, tmp);
#pragma unroll
    for (int v = 0; v < CW; ++v) be1[v] = tmp[v];
    be1[CW] = a.beta[1][i + CW];
  }
  wait_previous_grid();
  allow_next_grid();
  if (!live) return;
  const int sb = blockIdx.y * ck.spc, se = min(sb + ck.spc, n_shots);
  for (int s = sb; s < se; ++s) {
    const long long so = (long long)s * g.field;
    const T* __restrict__ pc = a.cur + so;
    const T* __restrict__ pp = a.prev + so;
    // the centre row with one chunk either side, the rows +-1, +-2 (x neighbours)
    T cm[CW], c0[CW], cp[CW], xm1[CW], xp1[CW], xm2[CW], xp2[CW], p0[CW];
    vldg<T, CW>(pc + i - CW, cm);
    vldg<T, CW>(pc + i, c0);
    vldg<T, CW>(pc + i + CW, cp);
    vldg<T, CW>(pc + i - ld, xm1);
    vldg<T, CW>(pc + i + ld, xp1);
    if (R == 2) {
      vldg<T, CW>(pc + i - 2 * ld, xm2);
      vldg<T, CW>(pc + i + 2 * ld, xp2);
    }
    vldg<T, CW>(pp + i, p0);
    T pm[CW], ppn[CW], pxm[CW], pxp[CW];  // adjoint: q^{k+2} beside the chunk, for the face sums
    if (ADJ) {
      vldg<T, CW>(pp + i - CW, pm);
      vldg<T, CW>(pp + i + CW, ppn);
      vldg<T, CW>(pp + i - ld, pxm);
      vldg<T, CW>(pp + i + ld, pxp);
    }
    T fo0[CW], fo0n[CW], fo1[CW], fo1n;
    vldg<T, CW>(a.f_old[0] + so + i, fo0);
    vldg<T, CW>(a.f_old[0] + so + i + ld, fo0n);
    vldg<T, CW>(a.f_old[1] + so + i, fo1);
    fo1n = a.f_old[1][so + i + CW];
    T lpin[CW], gr[CW];
    if (ADJ && a.lap) {
      vldg<T, CW>(a.lap + so + i, lpin);
      vload<T, CW>(a.grad + so + i, gr);
    }
    // the source stencil of this shot (forward)
    int bx = -4, bz = -4;
    if (!ADJ && a.src_corner) { bx = a.src_corner[2 * s]; bz = a.src_corner[2 * s + 1]; }
    auto zv = [&](const T (&row)[CW], int u) -> T {  // centre row, column zc + u, u in [-CW, 2 CW)
      return u < 0 ? cm[CW + u] : (u >= CW ? cp[u - CW] : row[u]);
    };
    auto pz = [&](int u) -> T { return u < 0 ? pm[CW + u] : (u >= CW ? ppn[u - CW] : p0[u]); };
    T out[CW], lout[CW], f0x[CW], f0z[CW], f1x[CW], f1z_last = T(0);
#pragma unroll
    for (int v = 0; v < CW; ++v) {
      const T c = c0[v];
      T lap = fma_rn(g.w1b, add_rn(zv(c0, v - 1), zv(c0, v + 1)), fma_rn(g.w1a, add_rn(xm1[v], xp1[v]), mul_rn(g.wc, c)));
      if (R == 2)
        lap = fma_rn(g.w2b, add_rn(zv(c0, v - 2), zv(c0, v + 2)), fma_rn(g.w2a, add_rn(xm2[v], xp2[v]), lap));
      T pml = T(0);
      f0x[v] = f1x[v] = f0z[v] = T(0);
      if (!core[v]) {
        // axis 0 (x): faces f = x (index i) and x + 1 (index i + ld)
        {
          const T h2 = a.hx2;
          T f0, f1;
          if (!ADJ) {
            f0 = fma_rn(be0[v], add_rn(c, -xm1[v]), mul_rn(al0[v], fo0[v]));
            f1 = fma_rn(be0n[v], add_rn(xp1[v], -c), mul_rn(al0n[v], fo0n[v]));
            pml = fma_rn(h2, add_rn(add_rn(f1, fo0n[v]), -add_rn(f0, fo0[v])), pml);
          } else {
            const T sm = add_rn(xm1[v], pxm[v]), s0 = add_rn(c, p0[v]), sp = add_rn(xp1[v], pxp[v]);
            f0 = fma_rn(-h2, add_rn(s0, -sm), mul_rn(al0[v], fo0[v]));
            f1 = fma_rn(-h2, add_rn(sp, -s0), mul_rn(al0n[v], fo0n[v]));
            pml = add_rn(pml, add_rn(mul_rn(be0n[v], f1), -mul_rn(be0[v], f0)));
          }
          f0x[v] = f0;
          f1x[v] = f1;
        }
        // axis 1 (z): faces f = z (index i + v) and z + 1
        {
          const T h2 = a.hz2;
          const T fon = v + 1 < CW ? fo1[v + 1] : fo1n;
          T f0, f1;
          if (!ADJ) {
            f0 = fma_rn(be1[v], add_rn(c, -zv(c0, v - 1)), mul_rn(al1[v], fo1[v]));
            f1 = fma_rn(be1[v + 1], add_rn(zv(c0, v + 1), -c), mul_rn(al1[v + 1], fon));
            pml = fma_rn(h2, add_rn(add_rn(f1, fon), -add_rn(f0, fo1[v])), pml);
          } else {
            const T sm = add_rn(zv(c0, v - 1), pz(v - 1)), s0 = add_rn(c, p0[v]), sp = add_rn(zv(c0, v + 1), pz(v + 1));
            f0 = fma_rn(-h2, add_rn(s0, -sm), mul_rn(al1[v], fo1[v]));
            f1 = fma_rn(-h2, add_rn(sp, -s0), mul_rn(al1[v + 1], fon));
            pml = add_rn(pml, add_rn(mul_rn(be1[v + 1], f1), -mul_rn(be1[v], f0)));
          }
          f0z[v] = f0;
          if (zc + v == g.n1 - 1) f1z_last = f1;
        }
      }
      const T av = core[v] ? T(1) : A[v], bv = core[v] ? T(1) : B[v], zz = core[v] ? T(0) : ZZ[v];
      if (!ADJ) {
        const T L = add_rn(lap, pml);
        lout[v] = L;
        T o = fma_rn(-zz, c, fma_rn(C[v], L, fma_rn(-bv, p0[v], add_rn(c, c))));
        const int dx = x - bx, dz = zc + v - bz;
        if (dx >= 0 && dx <= 1 && dz >= 0 && dz <= 1) o = add_rn(o, mul_rn(a.src_w[4 * s + 2 * dx + dz], a.wavelet[a.n]));
        out[v] = mul_rn(av, o);
      } else {
        const T o = fma_rn(-bv, p0[v], fma_rn(C[v], add_rn(lap, -pml), fma_rn(-zz, c, add_rn(c, c))));
        out[v] = a.apply_a ? mul_rn(av, o) : o;
        if (a.lap) gr[v] = fma_rn(c, lpin[v], gr[v]);
      }
    }
    // stores: whole chunks as vectors, partial chunks cell by cell; faces only where the cell is not
    // in the core box (the core box's faces are never written)
    bool any_core = false;
#pragma unroll
    for (int v = 0; v < CW; ++v) any_core = any_core || core[v];
    if (all_own) {
      vstore<T, CW>(a.next + so + i, out);
      if (!ADJ && a.lap_out) vstore<T, CW>(a.lap_out + so + i, lout);
      if (ADJ && a.lap) vstore<T, CW>(a.grad + so + i, gr);
      if (!any_core) {
        vstore<T, CW>(a.f_new[0] + so + i, f0x);
        vstore<T, CW>(a.f_new[1] + so + i, f0z);
        if (x == g.n0 - 1) vstore<T, CW>(a.f_new[0] + so + i + ld, f1x);
      }
    } else {
#pragma unroll
      for (int v = 0; v < CW; ++v) {
        if (!own[v]) continue;
        a.next[so + i + v] = out[v];
        if (!ADJ && a.lap_out) a.lap_out[so + i + v] = lout[v];
        if (ADJ && a.lap) a.grad[so + i + v] = gr[v];
        if (!core[v]) {
          a.f_new[0][so + i + v] = f0x[v];
          a.f_new[1][so + i + v] = f0z[v];
          if (x == g.n0 - 1) a.f_new[0][so + i + v + ld] = f1x[v];
        }
      }
    }
    if (all_own && any_core) {
#pragma unroll
      for (int v = 0; v < CW; ++v)
        if (!core[v]) {
          a.f_new[0][so + i + v] = f0x[v];
          a.f_new[1][so + i + v] = f0z[v];
          if (x == g.n0 - 1) a.f_new[0][so + i + v + ld] = f1x[v];
        }
    }
    if (g.n1 - 1 >= zc && g.n1 - 1 < zc + CW && own[g.n1 - 1 - zc < CW ? g.n1 - 1 - zc : 0] &&
        !core[g.n1 - 1 - zc < CW ? g.n1 - 1 - zc : 0])
      a.f_new[1][so + i + (g.n1 - zc)] = f1z_last;  // the last face of the row (first ghost column)
  }
}

}  // namespace nw
