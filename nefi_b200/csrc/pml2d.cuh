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
// has. The thread of cell (x, z) computes its own face and the next one (f = x, x+1), writes its own,
// and the last cell of a row or column also writes face P_ax. psi and Psi are double buffered by step
// parity, so no thread reads a face another thread of the same step writes.
#pragma once
#include "kernels.cuh"

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
};

// Thread t of shot s (grid.y) steps the t-th cell outside the tiled box, row by row: the rows above
// it, the strips left and right of it, the rows below it. CTAs past the last cell take the receiver
// samples of p^n on the forward's record steps (p^n is read-only in this step). Offsets inside a field
// are 32-bit (a field holds fewer than 2^31 elements).
constexpr int PML_THREADS = 256;

template <typename T, int R, bool ADJ>
__global__ void __launch_bounds__(PML_THREADS) pml2d_step(KGrid<T> g, PmlStep<T> a) {
  wait_previous_grid();
  allow_next_grid();
  const int s = blockIdx.y;
  const int top = a.kx0 * g.n1;
  const int bw = a.kz0 + (g.n1 - a.kz1);
  const int mid = (a.kx1 - a.kx0) * bw;
  const int n_layer = top + mid + (g.n0 - a.kx1) * g.n1;
  const int cell_ctas = (n_layer + PML_THREADS - 1) / PML_THREADS;
  if ((int)blockIdx.x >= cell_ctas) {  // the receiver samples
    const int r = ((int)blockIdx.x - cell_ctas) * PML_THREADS + threadIdx.x;
    if (!ADJ && a.traces && r < a.n_rec)
      a.traces[((long long)s * a.n_rec + r) * a.n_t + a.j] =
          sample_point<T, 4>(a.cur + (long long)s * g.field, a.rec_idx, a.rec_w, r);
    return;
  }
  const int t = blockIdx.x * PML_THREADS + threadIdx.x;
  if (t >= n_layer) return;
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
  const long long so = (long long)s * g.field;
  const T* __restrict__ pc = a.cur + so;
  const T* __restrict__ pp = a.prev + so;
  const int ld = (int)g.s0;
  const int row = (int)g.origin + x * ld;
  const bool core_row = x >= a.cx0 && x < a.cx1;
  {
    const int i = row + z;
    const T c = pc[i];
    // 5- or 9-point Laplacian in the reference's zero-padded convolution (fixed rounding sequence)
    T lap = fma_rn(g.w1b, add_rn(pc[i - 1], pc[i + 1]), fma_rn(g.w1a, add_rn(pc[i - ld], pc[i + ld]), mul_rn(g.wc, c)));
    if (R == 2)
      lap = fma_rn(g.w2b, add_rn(pc[i - 2], pc[i + 2]), fma_rn(g.w2a, add_rn(pc[i - 2 * ld], pc[i + 2 * ld]), lap));
    // the faces f = x, x+1 (axis 0, stride ld) and f = z, z+1 (axis 1, stride 1)
    T pml = T(0);  // forward: sum_ax (0.5/h) D-(psi_k + psi_{k-1});  adjoint: sum_ax D-(beta Psi_k)
    // Inside the core box the faces contribute exact zeros (forward: psi stays zero there, alpha = 1,
    // beta = 0; adjoint: beta = 0 multiplies the face cotangents) and A = B = 1, ZZ = 0, so the cell
    // takes the same rounding sequence with those constants and neither reads nor writes a face.
    const bool core = core_row && z >= a.cz0 && z < a.cz1;
#pragma unroll
    for (int ax = 0; ax < 2; ++ax) {
      if (core) break;
      const int st = ax == 0 ? ld : 1;
      const int j = i + st;  // index of face f+1
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
}

}  // namespace nw
