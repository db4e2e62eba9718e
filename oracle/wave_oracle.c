/*
 * wave_oracle.c — CPU oracle of NEFI's acoustic leapfrog propagator and its discrete adjoint.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * call this library, and only as the checker or the timed CPU baseline; the CUDA product path
 * never links or calls it.
 *
 * It restates, in plain C with one straightforward loop per operation, the algorithm of
 *   nefi/physics/wave.py:125-168   (Laplacian, zero outside the grid)
 *   nefi/physics/wave.py:520-554   (leapfrog step with sponge / Cerjan coefficients and sources)
 *   nefi/physics/wave.py:321-324, 699-750 (receiver sampling, forward run)
 *   nefi/physics/timestep.py:78-169 (time loop; sample 0 is the initial state)
 * and the exact discrete adjoint torch.autograd derives from those lines. Built in float64 (the
 * oracle proper) and float32 (to measure the effect of single precision). Parity of this file
 * with the reference is pinned by tests/test_oracle_golden.py against vectors produced by the
 * reference itself (tests/golden/make_golden.py).
 */
#include <stdlib.h>
#include <string.h>

typedef struct oracle_geom {
  int ndim;        /* 2 or 3 */
  int order;       /* 2 or 4 */
  long n[3];       /* padded extents */
  double w_center; /* Laplacian weights */
  double w1[3];
  double w2[3];
} oracle_geom;

static long oracle_cells(const oracle_geom* g) {
  return g->n[0] * g->n[1] * (g->ndim == 3 ? g->n[2] : 1);
}

#define REAL double
#define SFX _f64
#include "wave_oracle_impl.h"
#undef REAL
#undef SFX

#define REAL float
#define SFX _f32
#include "wave_oracle_impl.h"
#undef REAL
#undef SFX

int oracle_version(void) { return 1; }
