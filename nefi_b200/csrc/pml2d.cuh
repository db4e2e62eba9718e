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
// and C dJ/dC += q^{k+1} L_k with L_k stored by the forward step. The receiver cotangents of the
// cells outside the tiled box are added after the step, q^k += A C R^T g_k: by this launch when the
// host lists those cells for it, else by inject_kernel after the step, like the 3-D adjoint.
//
// Face f of axis ax (between cells f-1 and f, f = 0..P_ax) is stored at the cell index of f in the
// ghost layout: face P_ax lands in the first ghost row (x) or column (z), which the layout always
// has. The thread of cell (x, z) computes its own face and the next one (f = x, x+1), writes its own,
// and the last cell of a row or column also writes face P_ax. psi and Psi are double buffered by step
// parity, so no thread reads a face another thread of the same step writes.
#pragma once
#include "kernels.cuh"
#include "stencil2d.cuh"  // vector loads and stores

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
  // forward record steps: receiver samples of p^n, taken by extra CTAs of the same launch (NULL: none)
  T* __restrict__ traces;
  const int64_t* __restrict__ rec_idx;
  const T* __restrict__ rec_w;
  int n_rec, n_t, j;
  // adjoint: the gradient
  const T* __restrict__ lap;
  T* __restrict__ grad;            // per-shot accumulators of C dJ/dC
  // adjoint record steps: the receiver cotangents of the touched cells in the layer (ghost-layout
  // offsets lc_off, ascending, with their CSR rows lc_gid), added to the cells after the step as
  // inject_kernel does (NULL gtr: none)
  const T* __restrict__ gtr;
  const int* __restrict__ lc_off;
  const int* __restrict__ lc_gid;
  int n_lc;
  const int* __restrict__ gc_ptr;
  const int* __restrict__ gc_rec;
  const T* __restrict__ gc_w;
};

// Thread t of shot s (grid.y) steps the t-th 16-byte vector of W = 16 / sizeof(T) cells of the layer
// (the cells outside the tiled box), row by row: the rows above the box, the vectors left and right of
// it, the rows below it. Every cell takes the rounding sequence of the one-cell formulas above. A vector
// starts at a column that is a multiple of W (the box's first column is one), so with the ghost layout's
// 32-element rows and origin all its loads are aligned 16-byte loads; its lanes that lie in the box or
// past the last column are computed and not stored. The loads stay inside the level: the row pitch is a
// multiple of W at least P1 + R, so a vector never crosses a row, and only the centre row reads the
// neighbouring vectors (into the ghost row below at most). All loads come before any store, so the
// compiler may keep them in flight together. CTAs past the last vector take the receiver samples of p^n
// on the forward's record steps (p^n is read-only in this step). Offsets inside a field are 32-bit (a
// field holds fewer than 2^31 elements).
constexpr int PML_THREADS = 256;

// Vectors of the layer (outside the tiled box) of a P0 x P1 grid, W cells each.
__host__ __device__ __forceinline__ int pml_layer_vectors(int n0, int n1, int kx0, int kx1, int kz0, int kz1, int W) {
  const int nvr = (n1 + W - 1) / W;
  return (n0 - (kx1 - kx0)) * nvr + (kx1 - kx0) * (kz0 / W + nvr - kz1 / W);
}

template <typename T, int R, bool ADJ>
__global__ void __launch_bounds__(PML_THREADS) pml2d_step(KGrid<T> g, PmlStep<T> a) {
  constexpr int W = 16 / (int)sizeof(T);
  const int s = blockIdx.y;
  const int nvr = (g.n1 + W - 1) / W;
  const int vl = a.kz0 / W, vr0 = a.kz1 / W;
  const int bw = vl + (nvr - vr0);
  const int top = a.kx0 * nvr;
  const int mid = (a.kx1 - a.kx0) * bw;
  const int n_vec = top + mid + (g.n0 - a.kx1) * nvr;
  const int vec_ctas = (n_vec + PML_THREADS - 1) / PML_THREADS;
  if ((int)blockIdx.x >= vec_ctas) {  // the receiver samples
    wait_previous_grid();
    allow_next_grid();
    const int r = ((int)blockIdx.x - vec_ctas) * PML_THREADS + threadIdx.x;
    if (!ADJ && a.traces && r < a.n_rec)
      a.traces[((long long)s * a.n_rec + r) * a.n_t + a.j] =
          sample_point<T, 4>(a.cur + (long long)s * g.field, a.rec_idx, a.rec_w, r);
    return;
  }
  const int t = blockIdx.x * PML_THREADS + threadIdx.x;
  if (t >= n_vec) return;
  int x, m;
  if (t < top) {
    x = t / nvr;
    m = t - x * nvr;
  } else if (t < top + mid) {
    const int u = t - top;
    const int q = u / bw;
    const int r = u - q * bw;
    x = a.kx0 + q;
    m = r < vl ? r : vr0 + (r - vl);
  } else {
    const int u = t - top - mid;
    const int q = u / nvr;
    x = a.kx1 + q;
    m = u - q * nvr;
  }
  const int zb = m * W;
  const bool mid_row = x >= a.kx0 && x < a.kx1;
  const bool core_row = x >= a.cx0 && x < a.cx1;
  bool store[W], core[W];
  bool full = true;
#pragma unroll
  for (int v = 0; v < W; ++v) {
    const int z = zb + v;
    core[v] = core_row && z >= a.cz0 && z < a.cz1;
    store[v] = z < g.n1 && (!mid_row || z < a.kz0 || z >= a.kz1);
    full = full && store[v] && !core[v];
  }
  const int ld = (int)g.s0;
  const int i = (int)g.origin + x * ld + zb;

  // Constants of the sweep, loaded before the wait while the previous step finishes: face
  // coefficients at faces f (this vector) and f+1 (the next row; the next vector's first lane),
  // A, B, ZZ, C.
  T al0i[W], al0j[W], be0i[W], be0j[W], al1[W + 1], be1[W + 1], av[W], bv[W], zz[W], cc[W];
  vldg<T, W>(a.alpha[0] + i, al0i);
  vldg<T, W>(a.alpha[0] + i + ld, al0j);
  vldg<T, W>(a.beta[0] + i, be0i);
  vldg<T, W>(a.beta[0] + i + ld, be0j);
  {
    T t1[W], t2[W];
    vldg<T, W>(a.alpha[1] + i, t1);
    vldg<T, W>(a.beta[1] + i, t2);
#pragma unroll
    for (int v = 0; v < W; ++v) { al1[v] = t1[v]; be1[v] = t2[v]; }
    al1[W] = __ldg(a.alpha[1] + i + W);
    be1[W] = __ldg(a.beta[1] + i + W);
  }
  vldg<T, W>(a.A + i, av);
  vldg<T, W>(a.B + i, bv);
  vldg<T, W>(a.ZZ + i, zz);
  vldg<T, W>(a.C + i, cc);
  wait_previous_grid();
  allow_next_grid();

  const long long so = (long long)s * g.field;
  const T* __restrict__ pc = a.cur + so;
  const T* __restrict__ pp = a.prev + so;
  const T* __restrict__ fo0 = a.f_old[0] + so;
  const T* __restrict__ fo1 = a.f_old[1] + so;
  // the stencil field around the vector: centre row with its neighbour vectors, rows +-1, +-2
  T P[W], PL[W], PR[W], U1[W], D1[W], U2[W], D2[W], PPc[W];
  vload<T, W>(pc + i, P);
  vload<T, W>(pc + i - W, PL);
  vload<T, W>(pc + i + W, PR);
  vload<T, W>(pc + i - ld, U1);
  vload<T, W>(pc + i + ld, D1);
  if (R == 2) {
    vload<T, W>(pc + i - 2 * ld, U2);
    vload<T, W>(pc + i + 2 * ld, D2);
  }
  vload<T, W>(pp + i, PPc);
  T f0i[W], f0j[W], f1[W + 1];
  vload<T, W>(fo0 + i, f0i);
  vload<T, W>(fo0 + i + ld, f0j);
  {
    T t1[W];
    vload<T, W>(fo1 + i, t1);
#pragma unroll
    for (int v = 0; v < W; ++v) f1[v] = t1[v];
    f1[W] = fo1[i + W];
  }
  // adjoint: q^{k+2} at the x-neighbours and z-neighbours, the stored Laplacian and the accumulator
  T PU[W], PD[W], ppl = T(0), ppr = T(0), lp[W], gr[W];
  if (ADJ) {
    vload<T, W>(pp + i - ld, PU);
    vload<T, W>(pp + i + ld, PD);
    ppl = pp[i - 1];
    ppr = pp[i + W];
    if (a.lap) {
      vload<T, W>(a.lap + so + i, lp);
      vload<T, W>(a.grad + so + i, gr);
    }
  }
  int2 scor = make_int2(-1 << 20, -1 << 20);
  T swn = T(0);
  if (!ADJ && a.src_corner) {
    scor = make_int2(a.src_corner[2 * s], a.src_corner[2 * s + 1]);
    swn = a.wavelet[a.n];
  }

  auto zv = [&](int u) -> T { return u < 0 ? PL[W + u] : (u >= W ? PR[u - W] : P[u]); };
  T out[W], lout[W], n0f[W], n0l[W], n1f[W], e1 = T(0);  // n0l, e1: faces P0 / P1 (last row / column)
#pragma unroll
  for (int v = 0; v < W; ++v) {
    const T c = P[v];
    T lap = fma_rn(g.w1b, add_rn(zv(v - 1), zv(v + 1)), fma_rn(g.w1a, add_rn(U1[v], D1[v]), mul_rn(g.wc, c)));
    if (R == 2) lap = fma_rn(g.w2b, add_rn(zv(v - 2), zv(v + 2)), fma_rn(g.w2a, add_rn(U2[v], D2[v]), lap));
    T pml = T(0);
    T fx0, fx1, fz0, fz1;
    if (!ADJ) {  // psi_k = alpha psi_{k-1} + beta (p[f] - p[f-1])
      fx0 = fma_rn(be0i[v], add_rn(c, -U1[v]), mul_rn(al0i[v], f0i[v]));
      fx1 = fma_rn(be0j[v], add_rn(D1[v], -c), mul_rn(al0j[v], f0j[v]));
      T px = fma_rn(a.hx2, add_rn(add_rn(fx1, f0j[v]), -add_rn(fx0, f0i[v])), T(0));
      fz0 = fma_rn(be1[v], add_rn(c, -zv(v - 1)), mul_rn(al1[v], f1[v]));
      fz1 = fma_rn(be1[v + 1], add_rn(zv(v + 1), -c), mul_rn(al1[v + 1], f1[v + 1]));
      px = fma_rn(a.hz2, add_rn(add_rn(fz1, f1[v + 1]), -add_rn(fz0, f1[v])), px);
      if (!core[v]) pml = px;
    } else {  // Psi_k = alpha Psi_{k+1} - (0.5/h)(s[f] - s[f-1]),  s = q^{k+1} + q^{k+2}
      const T s0 = add_rn(c, PPc[v]);
      {
        const T sm = add_rn(U1[v], PU[v]), sp = add_rn(D1[v], PD[v]);
        fx0 = fma_rn(-a.hx2, add_rn(s0, -sm), mul_rn(al0i[v], f0i[v]));
        fx1 = fma_rn(-a.hx2, add_rn(sp, -s0), mul_rn(al0j[v], f0j[v]));
      }
      T px = add_rn(T(0), add_rn(mul_rn(be0j[v], fx1), -mul_rn(be0i[v], fx0)));
      {
        const T qm = v == 0 ? ppl : PPc[v - 1], qp = v == W - 1 ? ppr : PPc[v + 1];
        const T sm = add_rn(zv(v - 1), qm), sp = add_rn(zv(v + 1), qp);
        fz0 = fma_rn(-a.hz2, add_rn(s0, -sm), mul_rn(al1[v], f1[v]));
        fz1 = fma_rn(-a.hz2, add_rn(sp, -s0), mul_rn(al1[v + 1], f1[v + 1]));
      }
      px = add_rn(px, add_rn(mul_rn(be1[v + 1], fz1), -mul_rn(be1[v], fz0)));
      if (!core[v]) pml = px;
    }
    n0f[v] = fx0;
    n0l[v] = fx1;
    n1f[v] = fz0;
    if (zb + v == g.n1 - 1) e1 = fz1;
    const T A_ = core[v] ? T(1) : av[v], B_ = core[v] ? T(1) : bv[v], Z_ = core[v] ? T(0) : zz[v];
    T o;
    if (!ADJ) {
      const T L = add_rn(lap, pml);
      lout[v] = L;
      o = fma_rn(-Z_, c, fma_rn(cc[v], L, fma_rn(-B_, PPc[v], add_rn(c, c))));
      const int dx = x - scor.x, dz = zb + v - scor.y;
      if (dx >= 0 && dx <= 1 && dz >= 0 && dz <= 1) o = add_rn(o, mul_rn(a.src_w[4 * s + 2 * dx + dz], swn));
      out[v] = mul_rn(A_, o);
    } else {
      o = fma_rn(-B_, PPc[v], fma_rn(cc[v], add_rn(lap, -pml), fma_rn(-Z_, c, add_rn(c, c))));
      out[v] = a.apply_a ? mul_rn(A_, o) : o;
      if (a.lap) lout[v] = fma_rn(c, lp[v], gr[v]);
    }
  }

  if (ADJ && a.gtr) {  // the receiver cotangents of this vector's touched cells
    int lo = 0, hi = a.n_lc;
    while (lo < hi) {  // the first touched layer cell at or after the vector's first cell
      const int mid = (lo + hi) >> 1;
      if (a.lc_off[mid] < i) lo = mid + 1; else hi = mid;
    }
    const T* __restrict__ gs = a.gtr + (long long)s * a.n_rec * a.n_t + a.j;
    for (int e = lo; e < a.n_lc; ++e) {
      const int v = a.lc_off[e] - i;
      if (v >= W) break;
      const int gid = a.lc_gid[e];
      T acc = T(0);
      for (int q = a.gc_ptr[gid]; q < a.gc_ptr[gid + 1]; ++q)
        acc = fma_rn(a.gc_w[q], gs[(long long)a.gc_rec[q] * a.n_t], acc);
#pragma unroll
      for (int u = 0; u < W; ++u)
        if (u == v) out[u] = fma_rn(a.apply_a ? av[u] : T(1), mul_rn(cc[u], acc), out[u]);
    }
  }

  // stores: whole vectors where every lane is a non-core layer cell, else lane by lane
  T* __restrict__ fn0 = a.f_new[0] + so;
  T* __restrict__ fn1 = a.f_new[1] + so;
  T* __restrict__ lo = ADJ ? (a.lap ? a.grad + so : nullptr) : (a.lap_out ? a.lap_out + so : nullptr);
  if (full) {
    vstore<T, W>(a.next + so + i, out);
    if (lo) vstore<T, W>(lo + i, lout);
    vstore<T, W>(fn0 + i, n0f);
    vstore<T, W>(fn1 + i, n1f);
  } else {
#pragma unroll
    for (int v = 0; v < W; ++v) {
      if (!store[v]) continue;
      a.next[so + i + v] = out[v];
      if (lo) lo[i + v] = lout[v];
      if (!core[v]) {
        fn0[i + v] = n0f[v];
        fn1[i + v] = n1f[v];
      }
    }
  }
  // the last face of each axis: face P0 (ghost row P0) by the cells of the last row, face P1 (ghost
  // column P1) by the cell of the last column
  if (x == g.n0 - 1) {
#pragma unroll
    for (int v = 0; v < W; ++v)
      if (store[v] && !core[v]) fn0[i + ld + v] = n0l[v];
  }
#pragma unroll
  for (int v = 0; v < W; ++v)
    if (zb + v == g.n1 - 1 && store[v] && !core[v]) fn1[i + v + 1] = e1;
}

}  // namespace nw
