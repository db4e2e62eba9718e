/*
 * wave_oracle_impl.h — body of the CPU oracle, included once per scalar type by wave_oracle.c
 * with REAL (double/float) and SFX (_f64/_f32) defined.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA propagator, never a product path.
 *
 * Arrays are dense row-major padded grids (P0, P1[, P2]); values outside the grid read as zero.
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

/* Centred Laplacian with zero outside the padded grid (nefi/physics/wave.py:125-168). */
static void FN(lap_)(const oracle_geom* g, const REAL* p, REAL* out) {
  const long P0 = g->n[0], P1 = g->n[1], P2 = g->ndim == 3 ? g->n[2] : 1;
  const int R = g->order / 2;
  const long st[3] = {P1 * P2, P2, 1};
  const long ext[3] = {P0, P1, P2};
  for (long x = 0; x < P0; ++x)
    for (long y = 0; y < P1; ++y)
      for (long z = 0; z < P2; ++z) {
        const long i = (x * P1 + y) * P2 + z;
        const long pos[3] = {x, y, z};
        REAL acc = (REAL)g->w_center * p[i];
        for (int ax = 0; ax < g->ndim; ++ax) {
          for (int o = 1; o <= R; ++o) {
            const REAL w = (REAL)(o == 1 ? g->w1[ax] : g->w2[ax]);
            REAL pair = 0;
            if (pos[ax] - o >= 0) pair += p[i - o * st[ax]];
            if (pos[ax] + o < ext[ax]) pair += p[i + o * st[ax]];
            acc += w * pair;
          }
        }
        out[i] = acc;
      }
}

void FN(oracle_laplacian)(const oracle_geom* g, int n_fields, const REAL* p, REAL* out) {
  const long cells = oracle_cells(g);
  for (int f = 0; f < n_fields; ++f) FN(lap_)(g, p + f * cells, out + f * cells);
}

/*
 * Forward leapfrog run (nefi/physics/wave.py:520-554, 699-740; nefi/physics/timestep.py:140-149):
 *   p^{n+1} = A (2 p^n - B p^{n-1} + C Lap p^n + S w(n)),  B = 1 on the first step if first_b_one,
 * traces[s, r, j] = sum_k w_rk p^{j m}[idx_rk] (sample 0 is the initial state).
 * init_prev/init_cur: (n_shots, cells) or NULL for zeros. history (optional): (n_steps + 2,
 * n_shots, cells), level n at index n + 1.
 */
void FN(oracle_forward)(const oracle_geom* g, const REAL* C, const REAL* A, const REAL* B,
                        int first_b_one, int n_shots, const long* src_idx, const REAL* src_w,
                        int src_pts, const REAL* wavelet, int n_rec, int rec_pts,
                        const long* rec_idx, const REAL* rec_w, const REAL* init_prev,
                        const REAL* init_cur, int n_steps, int substeps, int n_t, REAL* traces,
                        REAL* history) {
  const long cells = oracle_cells(g);
#pragma omp parallel for schedule(static)
  for (int s = 0; s < n_shots; ++s) {
    REAL* buf = (REAL*)calloc(4 * cells, sizeof(REAL));
    REAL *pp = buf, *pc = buf + cells, *pn = buf + 2 * cells, *lp = buf + 3 * cells;
    if (init_prev) memcpy(pp, init_prev + s * cells, cells * sizeof(REAL));
    if (init_cur) memcpy(pc, init_cur + s * cells, cells * sizeof(REAL));
    if (history) {
      memcpy(history + ((long)0 * n_shots + s) * cells, pp, cells * sizeof(REAL));
      memcpy(history + ((long)1 * n_shots + s) * cells, pc, cells * sizeof(REAL));
    }
    for (int n = 0; n <= n_steps; ++n) {
      if (n % substeps == 0 && traces) {
        const int j = n / substeps;
        for (int r = 0; r < n_rec; ++r) {
          REAL acc = 0;
          for (int k = 0; k < rec_pts; ++k) acc += rec_w[r * rec_pts + k] * pc[rec_idx[r * rec_pts + k]];
          traces[((long)s * n_rec + r) * n_t + j] = acc;
        }
      }
      if (n == n_steps) break;
      FN(lap_)(g, pc, lp);
      for (long i = 0; i < cells; ++i) {
        const REAL b = (B && !(first_b_one && n == 0)) ? B[i] : (REAL)1;
        pn[i] = ((REAL)2 * pc[i] - b * pp[i]) + C[i] * lp[i];
      }
      if (src_idx) {
        const REAL wn = wavelet[n];
        for (int k = 0; k < src_pts; ++k) pn[src_idx[s * src_pts + k]] += src_w[s * src_pts + k] * wn;
      }
      if (A)
        for (long i = 0; i < cells; ++i) pn[i] = A[i] * pn[i];
      REAL* t = pp;
      pp = pc;
      pc = pn;
      pn = t;
      if (history) memcpy(history + ((long)(n + 2) * n_shots + s) * cells, pc, cells * sizeof(REAL));
    }
    free(buf);
  }
}

/*
 * Exact discrete adjoint of oracle_forward for trace cotangents g (n_shots, n_rec, n_t), from the
 * full history (the recursion torch.autograd performs through nefi/physics/wave.py:529-552):
 *   lambda^n = R^T g_n + 2 mu^{n+1} + Lap(C mu^{n+1}) - B mu^{n+2},  mu^n = A lambda^n (n >= 1),
 *   dJ/dC += mu^{n+1} Lap p^n.
 * Outputs per shot: grad_C (n_shots, cells), lambda0 (= dJ/dp^0) and mu1 (each may be NULL).
 */
void FN(oracle_adjoint)(const oracle_geom* g, const REAL* C, const REAL* A, const REAL* B,
                        int n_shots, int n_rec, int rec_pts, const long* rec_idx, const REAL* rec_w,
                        const REAL* history, int n_steps, int substeps, int n_t, const REAL* gtr,
                        REAL* grad_C, REAL* lambda0, REAL* mu1_out) {
  const long cells = oracle_cells(g);
  const int N = n_steps;
#pragma omp parallel for schedule(static)
  for (int s = 0; s < n_shots; ++s) {
    REAL* buf = (REAL*)calloc(6 * cells, sizeof(REAL));
    REAL *m2 = buf, *m1 = buf + cells, *m0 = buf + 2 * cells, *q = buf + 3 * cells,
         *lq = buf + 4 * cells, *lp = buf + 5 * cells;
    REAL* gc = grad_C + (long)s * cells;
    memset(gc, 0, cells * sizeof(REAL));
    for (int n = N; n >= 0; --n) {
      /* m1 = mu^{n+1}, m2 = mu^{n+2} */
      for (long i = 0; i < cells; ++i) q[i] = C[i] * m1[i];
      FN(lap_)(g, q, lq);
      for (long i = 0; i < cells; ++i) {
        const REAL b = B ? B[i] : (REAL)1;
        m0[i] = ((REAL)2 * m1[i] + lq[i]) - b * m2[i];
      }
      if (n % substeps == 0) {
        const int j = n / substeps;
        for (int r = 0; r < n_rec; ++r) {
          const REAL gv = gtr[((long)s * n_rec + r) * n_t + j];
          for (int k = 0; k < rec_pts; ++k) m0[rec_idx[r * rec_pts + k]] += rec_w[r * rec_pts + k] * gv;
        }
      }
      if (n <= N - 1) {
        const REAL* pn = history + ((long)(n + 1) * n_shots + s) * cells;
        FN(lap_)(g, pn, lp);
        for (long i = 0; i < cells; ++i) gc[i] += m1[i] * lp[i];
      }
      if (n == 0) {
        if (lambda0) memcpy(lambda0 + (long)s * cells, m0, cells * sizeof(REAL));
        if (mu1_out) memcpy(mu1_out + (long)s * cells, m1, cells * sizeof(REAL));
        break;
      }
      if (A)
        for (long i = 0; i < cells; ++i) m0[i] = A[i] * m0[i];
      REAL* t = m2;
      m2 = m1;
      m1 = m0;
      m0 = t;
    }
    free(buf);
  }
}

/*
 * 2-D PML run (nefi/physics/wave.py:476-501, 529-552), per shot, restating oracle.py's numpy
 * description of the same step in plain loops with the same operation order. Faces: psi_x has
 * (P0 + 1) x P1 entries (face f between cells f - 1 and f along x), psi_z P0 x (P1 + 1). With face
 * differences D+ (zero outside the grid) and cell differences D- of face arrays, step k:
 *   psi_k = alpha psi_{k-1} + beta D+ p^k,   L_k = Lap p^k + sum_ax (0.5/h) D-(psi_k + psi_{k-1}),
 *   p^{k+1} = A ((2 p^k - B p^{k-1}) + C L_k - ZZ p^k + S w(k)).
 * Lhist (optional): (n_steps, n_shots, cells), L_k at index k.
 */
void FN(oracle_pml_forward)(const oracle_geom* g, const REAL* C, const REAL* A, const REAL* B,
                            const REAL* ZZ, const REAL* alx, const REAL* bex, const REAL* alz,
                            const REAL* bez, REAL hx, REAL hz, int n_shots, const long* src_idx,
                            const REAL* src_w, int src_pts, const REAL* wavelet, int n_rec, int rec_pts,
                            const long* rec_idx, const REAL* rec_w, const REAL* init_prev,
                            const REAL* init_cur, int n_steps, int substeps, int n_t, REAL* traces,
                            REAL* Lhist) {
  const long P0 = g->n[0], P1 = g->n[1], cells = P0 * P1;
  const long fx = (P0 + 1) * P1, fz = P0 * (P1 + 1);
#pragma omp parallel for schedule(static)
  for (int s = 0; s < n_shots; ++s) {
    REAL* buf = (REAL*)calloc(4 * cells + 2 * fx + 2 * fz, sizeof(REAL));
    REAL *pp = buf, *pc = buf + cells, *pn = buf + 2 * cells, *L = buf + 3 * cells;
    REAL *psx = buf + 4 * cells, *nsx = psx + fx, *psz = nsx + fx, *nsz = psz + fz;
    if (init_prev) memcpy(pp, init_prev + s * cells, cells * sizeof(REAL));
    if (init_cur) memcpy(pc, init_cur + s * cells, cells * sizeof(REAL));
    for (int n = 0; n <= n_steps; ++n) {
      if (n % substeps == 0 && traces) {
        const int j = n / substeps;
        for (int r = 0; r < n_rec; ++r) {
          REAL acc = 0;
          for (int k = 0; k < rec_pts; ++k) acc += rec_w[r * rec_pts + k] * pc[rec_idx[r * rec_pts + k]];
          traces[((long)s * n_rec + r) * n_t + j] = acc;
        }
      }
      if (n == n_steps) break;
      FN(lap_)(g, pc, L);
      /* x faces */
      for (long f = 0; f <= P0; ++f)
        for (long z = 0; z < P1; ++z) {
          const long i = f * P1 + z;
          const REAL hi = f < P0 ? pc[f * P1 + z] : (REAL)0, lo = f > 0 ? pc[(f - 1) * P1 + z] : (REAL)0;
          nsx[i] = alx[i] * psx[i] + bex[i] * (hi - lo);
        }
      for (long x = 0; x < P0; ++x)
        for (long z = 0; z < P1; ++z) {
          const long i = x * P1 + z;
          L[i] = L[i] + ((nsx[i + P1] + psx[i + P1]) - (nsx[i] + psx[i])) * hx;
        }
      /* z faces */
      for (long x = 0; x < P0; ++x)
        for (long f = 0; f <= P1; ++f) {
          const long i = x * (P1 + 1) + f;
          const REAL hi = f < P1 ? pc[x * P1 + f] : (REAL)0, lo = f > 0 ? pc[x * P1 + f - 1] : (REAL)0;
          nsz[i] = alz[i] * psz[i] + bez[i] * (hi - lo);
        }
      for (long x = 0; x < P0; ++x)
        for (long z = 0; z < P1; ++z) {
          const long i = x * (P1 + 1) + z;
          L[x * P1 + z] = L[x * P1 + z] + ((nsz[i + 1] + psz[i + 1]) - (nsz[i] + psz[i])) * hz;
        }
      if (Lhist) memcpy(Lhist + ((long)n * n_shots + s) * cells, L, cells * sizeof(REAL));
      for (long i = 0; i < cells; ++i) pn[i] = (((REAL)2 * pc[i] - B[i] * pp[i]) + C[i] * L[i]) - ZZ[i] * pc[i];
      if (src_idx) {
        const REAL wn = wavelet[n];
        for (int k = 0; k < src_pts; ++k) pn[src_idx[s * src_pts + k]] += src_w[s * src_pts + k] * wn;
      }
      for (long i = 0; i < cells; ++i) pn[i] = A[i] * pn[i];
      REAL* t = pp; pp = pc; pc = pn; pn = t;
      t = psx; psx = nsx; nsx = t;
      t = psz; psz = nsz; nsz = t;
    }
    free(buf);
  }
}

/*
 * Exact discrete adjoint of oracle_pml_forward (derived by hand: D+^T = -D-, D-^T = -D+), with
 * mu^k = A lambda^k and face cotangents Psi:
 *   Psi_k    = alpha Psi_{k+1} - (0.5/h) D+(C mu^{k+1} + C mu^{k+2}),
 *   lambda^k = R^T g_k + (2 mu^{k+1} - ZZ mu^{k+1}) + Lap(C mu^{k+1}) - sum_ax D-(beta Psi_k) - B mu^{k+2},
 *   dJ/dC   += mu^{k+1} L_k  (L_k from the forward's Lhist).
 * Outputs per shot like oracle_adjoint.
 */
void FN(oracle_pml_adjoint)(const oracle_geom* g, const REAL* C, const REAL* A, const REAL* B,
                            const REAL* ZZ, const REAL* alx, const REAL* bex, const REAL* alz,
                            const REAL* bez, REAL hx, REAL hz, int n_shots, int n_rec, int rec_pts,
                            const long* rec_idx, const REAL* rec_w, const REAL* Lhist, int n_steps,
                            int substeps, int n_t, const REAL* gtr, REAL* grad_C, REAL* lambda0,
                            REAL* mu1_out) {
  const long P0 = g->n[0], P1 = g->n[1], cells = P0 * P1;
  const long fx = (P0 + 1) * P1, fz = P0 * (P1 + 1);
  const int N = n_steps;
#pragma omp parallel for schedule(static)
  for (int s = 0; s < n_shots; ++s) {
    REAL* buf = (REAL*)calloc(6 * cells + fx + fz, sizeof(REAL));
    REAL *m2 = buf, *m1 = buf + cells, *lam = buf + 2 * cells, *q = buf + 3 * cells,
         *s2 = buf + 4 * cells, *lq = buf + 5 * cells;
    REAL *Px = buf + 6 * cells, *Pz = Px + fx;
    REAL* gc = grad_C + (long)s * cells;
    memset(gc, 0, cells * sizeof(REAL));
    for (int k = N; k >= 0; --k) {
      for (long i = 0; i < cells; ++i) lam[i] = 0;
      if (k <= N - 1) {
        for (long i = 0; i < cells; ++i) {
          q[i] = C[i] * m1[i];
          s2[i] = q[i] + C[i] * m2[i];
        }
        for (long f = 0; f <= P0; ++f)
          for (long z = 0; z < P1; ++z) {
            const long i = f * P1 + z;
            const REAL hi = f < P0 ? s2[f * P1 + z] : (REAL)0, lo = f > 0 ? s2[(f - 1) * P1 + z] : (REAL)0;
            Px[i] = alx[i] * Px[i] - hx * (hi - lo);
          }
        for (long x = 0; x < P0; ++x)
          for (long f = 0; f <= P1; ++f) {
            const long i = x * (P1 + 1) + f;
            const REAL hi = f < P1 ? s2[x * P1 + f] : (REAL)0, lo = f > 0 ? s2[x * P1 + f - 1] : (REAL)0;
            Pz[i] = alz[i] * Pz[i] - hz * (hi - lo);
          }
        FN(lap_)(g, q, lq);
        for (long i = 0; i < cells; ++i) lam[i] = ((REAL)2 * m1[i] - ZZ[i] * m1[i]) + lq[i];
        for (long x = 0; x < P0; ++x)
          for (long z = 0; z < P1; ++z) {
            const long i = x * P1 + z;
            lam[i] = lam[i] - (bex[i + P1] * Px[i + P1] - bex[i] * Px[i]);
          }
        for (long x = 0; x < P0; ++x)
          for (long z = 0; z < P1; ++z) {
            const long i = x * (P1 + 1) + z;
            lam[x * P1 + z] = lam[x * P1 + z] - (bez[i + 1] * Pz[i + 1] - bez[i] * Pz[i]);
          }
        for (long i = 0; i < cells; ++i) lam[i] = lam[i] - B[i] * m2[i];
        const REAL* Lk = Lhist + ((long)k * n_shots + s) * cells;
        for (long i = 0; i < cells; ++i) gc[i] += m1[i] * Lk[i];
      }
      if (k % substeps == 0) {
        const int j = k / substeps;
        for (int r = 0; r < n_rec; ++r) {
          const REAL gv = gtr[((long)s * n_rec + r) * n_t + j];
          for (int c = 0; c < rec_pts; ++c) lam[rec_idx[r * rec_pts + c]] += rec_w[r * rec_pts + c] * gv;
        }
      }
      if (k == 0) {
        if (lambda0) memcpy(lambda0 + (long)s * cells, lam, cells * sizeof(REAL));
        if (mu1_out) memcpy(mu1_out + (long)s * cells, m1, cells * sizeof(REAL));
        break;
      }
      REAL* t = m2; m2 = m1; m1 = t;
      for (long i = 0; i < cells; ++i) m1[i] = A[i] * lam[i];
    }
    free(buf);
  }
}

#undef FN
#undef CAT
#undef CAT_
