/*
 * nefi_wave.h — C ABI of the B200 (sm_100a) acoustic leapfrog propagator and its exact adjoint.
 *
 * The library replaces the time loop of NEFI's wave operators: the leapfrog step
 * `_LeapfrogBase._step_fn` (nefi/physics/wave.py:520-554), the loop driver `run_timestepping`
 * (nefi/physics/timestep.py:78-169), receiver sampling `_sample` (nefi/physics/wave.py:321-324),
 * source injection (nefi/physics/wave.py:715-721), and the reverse-mode autodiff of all of them
 * (the discrete adjoint NEFI obtains from torch.autograd, nefi/physics/wave.py:46-49).
 *
 * Conventions
 *  - Every pointer is a device pointer unless stated otherwise; sizes are element counts.
 *  - Device buffers holding fields (medium, storage, adjoint work levels, accumulators) start on
 *    16-byte boundaries: the kernels move fields in 16-byte vectors. nw_forward / nw_adjoint return
 *    NW_ERR_ARG for a buffer that does not.
 *  - Nothing is allocated by the library: the caller passes every buffer, sized by the
 *    nw_*_bytes() queries. The library never frees caller memory.
 *  - All work is enqueued on `stream` (a cudaStream_t passed as void*); calls are asynchronous
 *    unless they say otherwise. Calls on distinct streams with distinct buffers may overlap.
 *  - Return value: NW_OK or an NW_ERR_* code; nw_last_error() gives a message for the calling
 *    thread's last failure.
 *  - Grid arrays ("fields") use the ghost layout described by nw_grid: the padded simulation grid
 *    (P0[,P1],Pl), last axis contiguous, surrounded by zero cells so that every stencil read is in
 *    bounds and reads zero outside the grid (the reference's zero-padded convolution,
 *    nefi/physics/wave.py:144-168). The library writes only interior cells, so the ghost cells of
 *    a buffer that started zeroed stay zero.
 */
#ifndef NEFI_WAVE_H
#define NEFI_WAVE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NW_ABI_VERSION 6

/* scalar type of a computation */
enum { NW_F32 = 0, NW_F64 = 1 };
/* absorbing layer kind (nefi/physics/wave.py:80, 469-501); NW_ABS_PML is 2-D only */
enum { NW_ABS_NONE = 0, NW_ABS_SPONGE = 1, NW_ABS_CERJAN = 2, NW_ABS_PML = 3 };
/* snapshot encodings for checkpointed gradients */
enum { NW_SNAP_EXACT = 0, NW_SNAP_F16 = 1, NW_SNAP_BF16 = 2, NW_SNAP_I16 = 3, NW_SNAP_D16 = 4 };
/* status codes */
enum {
  NW_OK = 0,
  NW_ERR_ARG = 1,         /* invalid argument (the message names it) */
  NW_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  NW_ERR_UNSUPPORTED = 3, /* valid but not built (dimension/order/absorbing combination) */
  NW_ERR_NONFINITE = 4,   /* a snapshot block held a non-finite value or scale */
  NW_ERR_TIMEOUT = 5      /* a bounded device-side wait gave up */
};

/*
 * Geometry of one padded grid. The caller fills ndim, order, dtype, absorbing, n[], core_lo[],
 * core_hi[] and the stencil weights; nw_grid_layout() fills the layout fields.
 * Replaces WaveGrid (nefi/physics/wave.py:195-318) and laplacian_kernel (wave.py:125-141).
 */
typedef struct nw_grid {
  int32_t ndim;       /* 2 or 3 */
  int32_t order;      /* 2 or 4: spatial accuracy of the Laplacian */
  int32_t dtype;      /* NW_F32 or NW_F64 */
  int32_t absorbing;  /* NW_ABS_* */
  int32_t n[3];       /* padded extents P per axis; the last used axis is contiguous */
  int32_t core_lo[3]; /* cells with lo <= i < hi on every axis are outside the layer */
  int32_t core_hi[3];
  double w_center;    /* Laplacian weights: centre, +-1 and +-2 neighbours per axis */
  double w1[3];
  double w2[3];
  /* --- filled by nw_grid_layout --- */
  int32_t radius;      /* stencil radius: order / 2 */
  int32_t guard;       /* zero elements before the first storage row (keeps 16-byte tile copies
                          that start left of column 0 inside the buffer) */
  int64_t stride[3];   /* element strides per axis in the ghost layout */
  int64_t origin;      /* element offset of cell (0,..,0) */
  int64_t field_elems; /* elements per field buffer, ghosts included (a multiple of 32) */
} nw_grid;

/* Fills radius/guard/stride/origin/field_elems of `g`. Host only, no CUDA call. */
int nw_grid_layout(nw_grid* g);

/*
 * Launch shape of the 2-D step kernels, forward and adjoint separately: a CTA owns a tile of
 * 8*rx rows by 32*vz columns and loops over shots_per_cta shots. Zero fields take the library's
 * defaults. 3-D grids ignore it.
 */
typedef struct nw_tuning {
  int32_t vz;                /* forward: columns per thread, 2 or 4 (float32), 2 (float64) */
  int32_t rx;                /* forward: rows per thread, 2, 4 or 8 */
  int32_t shots_per_cta;     /* forward: shots per CTA, >= 1 */
  int32_t adj_vz;            /* the same for the adjoint steps; adj_shots_per_cta shots share */
  int32_t adj_rx;            /*   one gradient accumulator field */
  int32_t adj_shots_per_cta;
  int32_t depth;             /* forward steps per launch: 1 (0 = 1) or 2 (2-D without a PML, and a
                                ring of four levels, nw_storage.ring_levels = 4); two steps per launch
                                give bitwise the fields of one. With depth 2 the forward tile of
                                nw_tile_shape is the core a launch stores: (8*rx - 2*radius) rows by
                                (32*vz - 2*(16 / element size)) columns */
  int32_t reserved;
} nw_tuning;

/*
 * Resolves the defaults of `t` for grid `g` in place and reports the tile shapes:
 * shape = {forward rows, forward columns, adjoint rows, adjoint columns}.
 */
int nw_tile_shape(const nw_grid* g, nw_tuning* t, int32_t* shape);

/*
 * Number of gradient accumulator fields (in the grid's dtype) nw_adjoint fills for n_shots
 * shots: one per shot in 3-D and with a PML, one per group of adj_shots_per_cta shots otherwise.
 */
int nw_adjoint_groups(const nw_grid* g, const nw_tuning* t, int32_t n_shots);

/*
 * Point stencils of one acquisition. Sources: one multilinear stencil per shot, injected as
 * weight[k] * wavelet[n] into cell corner + bits(k) every step n (nefi/physics/wave.py:312-318,
 * 715-721). Receivers: one multilinear stencil per receiver, shared by all shots, sampled at
 * every record step (nefi/physics/wave.py:272-300, 321-324, 723-729).
 * The adjoint of the receiver sampling is given as a cell-major table (CSR over the cells the
 * receivers touch) so that the adjoint injection sums each cell in a fixed order.
 * For 2-D grids the per-tile tables index the same data by the tile shape nw_tile_shape reports.
 */
typedef struct nw_acquisition {
  int32_t n_shots;
  int32_t has_source;          /* 0 for the initial-value (photoacoustic) operator */
  const int32_t* src_corner;   /* (n_shots, ndim) lower corner cell */
  const void* src_weight;      /* (n_shots, 2^ndim) dtype: w / cell_volume * dt^2 */
  const void* wavelet;         /* (n_steps,) dtype: source time function at t = n dt */
  int32_t n_rec;
  int32_t n_cells;             /* cells touched by the receiver stencils */
  const int64_t* rec_index;    /* (n_rec, 2^ndim) ghost-layout offsets */
  const void* rec_weight;      /* (n_rec, 2^ndim) dtype */
  const int64_t* cell_index;   /* (n_cells,) ghost-layout offsets, ascending */
  const int32_t* cell_ptr;     /* (n_cells + 1,) CSR row pointers into cell_rec/cell_weight */
  const int32_t* cell_rec;     /* receiver id per entry */
  const void* cell_weight;     /* dtype weight per entry */
  /* 2-D per-tile tables (tiles in row-major order, tiles_z along the contiguous axis): receivers
     by the forward tile shape, receiver-touched cells by the adjoint tile shape */
  int32_t tiles_z;
  int32_t tile_rows, tile_cols;    /* forward tile shape the receiver tables were built for */
  const int32_t* rec_corner;       /* (n_rec, 2) corner cell of each receiver stencil */
  const int32_t* tile_rec_ptr;     /* (n_tiles + 1): receivers whose corner lies in the tile */
  const int32_t* tile_rec_list;
  int32_t adj_tiles_z;
  int32_t adj_tile_rows, adj_tile_cols;  /* adjoint tile shape the cell tables were built for */
  const int32_t* tile_cell_ptr;    /* (n_adj_tiles + 1): touched cells of the tile */
  const int32_t* tile_cell_local;  /* (x - x0) * adj_tile_cols + (z - z0) */
  const int32_t* tile_cell_gid;    /* row in cell_index / cell_ptr */
  /* 2-D PML only: 1 when the adjoint tile tables above were built for the tiles of the PML's tiled
     interior box (the adjoint tile grid starts at cell adj_box_corner = (x, z), the box's corner as
     the library derives it from medium.pml_core and the adjoint tile shape) and hold the
     receiver-touched cells inside it, while the n_layer_cells touched cells outside it are listed in
     layer_cell_index / layer_cell_gid: the box's adjoint launch and the layer's then add the receiver
     cotangents themselves. 0: the tables cover the whole grid from cell (0, 0), and a separate launch
     adds the cotangents after each PML step. */
  int32_t adj_tables_box;
  int32_t adj_box_corner[2];
  int32_t n_layer_cells;
  const int32_t* layer_cell_index; /* (n_layer_cells,) ghost-layout offsets, ascending */
  const int32_t* layer_cell_gid;   /* row in cell_index / cell_ptr */
} nw_acquisition;

/* The medium: c^2 dt^2 on the padded grid and the absorbing coefficients. */
typedef struct nw_medium {
  const void* c2dt2;  /* field (ghost layout) */
  const void* coef_a; /* field: A = 1/(1 + sigma dt/2) (sponge), 1/(1 + dt/2 sum zeta) (PML) or the
                         Cerjan taper; NULL if none */
  const void* coef_b; /* field: B = 1 - sigma dt/2 (sponge), 1 - dt/2 sum zeta (PML) or the Cerjan
                         taper; NULL if none */
  /* PML only (nefi/physics/wave.py:476-501), NULL otherwise: ZZ = dt^2 zeta_x zeta_z on cells, and
     per axis the face coefficients alpha = (1 - dt/2 zeta_f)/(1 + dt/2 zeta_f) and
     beta = dt (zeta_other - zeta_f)/((1 + dt/2 zeta_f) h), face f of an axis stored at the cell
     index f (face P_ax in the first ghost row / column) */
  const void* pml_zz;
  const void* pml_alpha[2];
  const void* pml_beta[2];
  double pml_half_inv_h[2];  /* 0.5 / h per axis: the factor of the psi divergence */
  int32_t pml_core[4];       /* x0, x1, z0, z1: a box of padded cells where every PML term vanishes
                                exactly (A = B = 1, ZZ = 0, and alpha = 1, beta = 0 on both faces of
                                both axes); the step skips the face fields there. All 0: no box */
} nw_medium;

/* Time axis: n_steps = (n_t - 1) * substeps; trace sample j is the state after j*substeps steps. */
typedef struct nw_time {
  int32_t n_steps;
  int32_t substeps;
  int32_t n_t;
  int32_t first_b_one; /* 1: the first step uses B = 1 on p^-1 (Cerjan, nefi/physics/wave.py:550-551) */
} nw_time;

/*
 * Wavefield storage. The pressure always advances through `ring`: three levels (four with
 * ring_levels = 4), level n at ring + ((n+1) % levels) * level_stride (level_stride = n_shots *
 * field_elems). What the gradient
 * needs of the forward run is Lap p^n for n = 0..N-1, the factor of the velocity term
 * mu^{n+1} * Lap p^n; it is kept in one of two ways.
 *  history != NULL: the forward step n stores Lap p^n at history + n*level_stride (N levels,
 *    grad_mode="autograd").
 *  history == NULL and snap != NULL: checkpointing (grad_mode="checkpoint",
 *    nefi/physics/timestep.py:141-169): the pair (p^{n0-1}, p^{n0}) is encoded into snapshot
 *    j = n0 / segment for every segment start n0; the adjoint decodes it into the ring and
 *    recomputes Lap p^{n0..n0+segment-1} into `segbuf` (segment levels). snap_kind selects exact
 *    copies or 16-bit values with one float scale per block of NW_SNAP_BLOCK elements: fp16 /
 *    bf16 with a power-of-two scale, or int16 mantissas scaled by the block maximum (NW_SNAP_I16,
 *    block floating point), or (NW_SNAP_D16) int16 codes of the second differences along the
 *    contiguous axis of integer values relative to a float anchor, with a float step per block
 *    (element z = anchor + step * Q[z]; the step is 1/32000 of the block's largest second
 *    difference, so the error of a smooth field is several times below NW_SNAP_I16's). The 16-bit
 *    kinds store p^{n0} and p^{n0} - p^{n0-1}.
 *  both NULL: forward only.
 */
#define NW_SNAP_BLOCK 32
typedef struct nw_storage {
  void* history;       /* N levels of Lap p^n, or NULL */
  void* ring;          /* 3 levels of p, always required */
  void* snap;          /* snapshot pool, nw_snapshot_bytes() bytes */
  void* segbuf;        /* `segment` levels of Lap p^n, used when snap != NULL */
  int32_t segment;     /* steps per checkpoint segment */
  int32_t snap_kind;   /* NW_SNAP_* */
  void* pml_psi;       /* PML only: 4 levels (axis x {even, odd step}), each n_shots fields, zero
                          before step 0: the auxiliary face fields psi. With snapshots the
                          snapshots also hold the two face fields each segment starts from, and
                          nw_adjoint re-runs segments in these levels */
  /* Binomial checkpointing (optional; both NULL: segment j's start goes into snapshot slot j and the
     adjoint decodes slot j for segment j). HOST memory, read during the calls: */
  const int32_t* snap_slot; /* per segment j: the slot nw_forward encodes its start state into, or -1 */
  const int32_t* schedule;  /* the adjoint's program: n_schedule triples (op, x, y), executed in order;
                               NW_SCHED_RESTORE (slot, j): decode slot `slot`, the state at segment j's
                               start; NW_SCHED_ADVANCE (j0, j1): forward steps from segment j0's start
                               to j1's, storing nothing; NW_SCHED_TAKE (slot, j): encode the state at
                               segment j's start (the ring's) into `slot`; NW_SCHED_YOUTURN (j, 0):
                               recompute segment j's Lap p levels from the state the ring holds at its
                               start, then run its adjoint steps. The segments are reversed last to
                               first, each by one YOUTURN. The batched calls ignore both fields */
  int32_t n_schedule;
  int32_t ring_levels;      /* levels in `ring`: 3 (0 means 3) or 4; level n at ring + ((n+1) % levels) *
                               level_stride. Four let the forward advance two steps per launch */
} nw_storage;
enum { NW_SCHED_RESTORE = 1, NW_SCHED_ADVANCE = 2, NW_SCHED_TAKE = 3, NW_SCHED_YOUTURN = 4 };

/* Bytes of one snapshot pool for `n_snap` snapshots of n_shots shots (both levels, and with a PML
 * the two face fields). */
size_t nw_snapshot_bytes(const nw_grid* g, int32_t n_shots, int32_t n_snap, int32_t snap_kind);

/*
 * Prepare the medium: c (physical grid, contiguous, dtype) -> c2dt2 = pad_replicate(c)^2 * dt2
 * in the ghost layout (nefi/physics/wave.py:222-240, 718). `n_abs` (host) is the layer width per axis.
 */
int nw_prepare_medium(const nw_grid* g, const int32_t* n_abs, const void* c, double dt2,
                      void* c2dt2, void* stream);

/*
 * Copy per-shot physical fields (n_shots, n...) into ghost-layout levels with a zero layer
 * (WaveGrid.pad(.., "zeros"), nefi/physics/wave.py:226-230) and form
 * p^-1 = p^0 + 1/2 c2dt2 * Lap p^0 (nefi/physics/wave.py:849-850).
 * Writes level p^0 into `p0_level` and p^-1 into `pm1_level` (each n_shots fields).
 */
int nw_initial_state(const nw_grid* g, const int32_t* n_abs, const nw_medium* m, int32_t n_shots,
                     const void* p0, void* pm1_level, void* p0_level, void* stream);

/*
 * Forward run of steps [n_begin, n_end) for all shots through the ring of `st`; with a history,
 * step n also stores Lap p^n there. Receiver samples of every recorded level
 * n in [n_begin, n_end) go to traces (n_shots, n_rec, n_t), and of level n_end when it is the last
 * step; with checkpointing, snapshots of every segment start in [n_begin, n_end) are encoded.
 * On entry ring levels n_begin-1 and n_begin must be in place. `tune` may be NULL.
 * With the PML and an interior box of at least one tile, each step forks its layer kernel onto a
 * second stream of the calling thread and joins it back into `stream` (also in nw_adjoint and the
 * batched sweeps); the first such call on a thread and device creates that stream and two events,
 * in relaxed capture mode, and keeps them until the process exits.
 * Replaces WaveOperator.simulate / run_timestepping (nefi/physics/wave.py:699-740,
 * nefi/physics/timestep.py:144-149).
 */
int nw_forward(const nw_grid* g, const nw_medium* m, const nw_acquisition* a, const nw_time* t,
               const nw_storage* st, const nw_tuning* tune, int32_t n_begin, int32_t n_end,
               void* traces, void* stream);

/*
 * Adjoint run for all shots: from trace cotangents `grad_traces` (n_shots, n_rec, n_t) computes
 *  - grad_acc: nw_adjoint_groups() fields in the grid's dtype (zeroed by the call) whose sum is
 *    c2dt2 * sum_shots sum_n mu^{n+1} * Lap p^n, i.e. c2dt2 times the gradient w.r.t. c2dt2
 *    (nw_reduce_grad_c divides the factor out), and
 *  - lambda0 / mu1 (n_shots fields each, may be NULL): the sensitivities of p^0 and A*p^1
 *    needed by the initial-value operator.
 * The steps advance q = c2dt2 * mu, which obeys the forward recursion with the source replaced
 * by c2dt2 * R^T g_n; `work` holds three q levels (3 * n_shots fields; 7 * n_shots with a PML, whose
 * adjoint also carries the face cotangents of psi, 2 axes x 2 levels). Uses the history or
 * recomputes segments from the snapshots in `st`. This is the discrete adjoint torch.autograd
 * derives from nefi/physics/wave.py:529-552 and nefi/physics/timestep.py:151-169.
 */
int nw_adjoint(const nw_grid* g, const nw_medium* m, const nw_acquisition* a, const nw_time* t,
               const nw_storage* st, const nw_tuning* tune, const void* grad_traces, void* work,
               void* grad_acc, void* lambda0, void* mu1, void* stream);

/*
 * Reduce gradient accumulators (n_acc fields in the grid's dtype holding c2dt2 * dJ/dc2dt2, as
 * nw_adjoint leaves them) in float64 and apply the chain rule of c2dt2 = pad_replicate(c)^2 dt^2: grad_c (physical
 * grid, float64) = pad_replicate^T(2 c_pad dt2 * sum_acc g / (c_pad^2 dt2))
 * (nefi/physics/wave.py:231-240, 718).
 * `accumulate` != 0 adds into grad_c instead of overwriting it.
 */
int nw_reduce_grad_c(const nw_grid* g, const int32_t* n_abs, const void* c, double dt2,
                     int32_t n_acc, const void* grad_acc, int32_t accumulate, double* grad_c,
                     void* stream);

/*
 * Gradient of the initial-value operator w.r.t. p0 (n_shots physical fields, dtype):
 * lambda^0 + lambda^-1 + Lap(1/2 c2dt2 lambda^-1) cropped to the physical grid, with
 * lambda^-1 = -B0 mu^1 (B0 = 1 when time.first_b_one). If grad_acc != NULL also adds
 * c2dt2 * 1/2 lambda^-1 * Lap p^0 of shot s to accumulator s / shots_per_acc (the c-dependence
 * of p^-1, nefi/physics/wave.py:850, in the accumulators' c2dt2-scaled convention).
 */
int nw_initial_state_adjoint(const nw_grid* g, const int32_t* n_abs, const nw_medium* m,
                             const nw_time* t, int32_t n_shots, const void* lambda0,
                             const void* mu1, const void* p0_level, void* grad_p0,
                             void* grad_acc, int32_t shots_per_acc, void* stream);

/*
 * Allocation-free gradient: the work of nw_adjoint followed by nw_reduce_grad_c (overwriting
 * grad_c), with the adjoint's scratch -- the adjoint levels and the gradient accumulators (in the
 * computation's dtype) -- taken
 * from one fixed array that the library holds in device memory instead of from caller buffers.
 * This entry point has no counterpart in the reference; it exists for callers that cannot allocate
 * device memory themselves: a host runtime that reaches this library only through the C ABI and
 * owns no CUDA allocator (a JVM or Go service binding it through JNI or cgo), a service that
 * reserves its device memory at start-up and may not allocate afterwards, or a latency-bound loop
 * that must not call cudaMalloc, which synchronises the device. The caller still passes every
 * input and the output grad_c (physical grid, float64).
 *  - Limit: 3 * n_shots * field_elems * sizeof(dtype) (7 * ... with a PML), rounded up to 256 bytes, plus
 *    nw_adjoint_groups() * field_elems * sizeof(dtype) bytes must not exceed NW_NOALLOC_SCRATCH_BYTES (64 MiB);
 *    e.g. 16 float32 shots on a 552^2 padded grid fit, 20 do not. Larger requests return
 *    NW_ERR_ARG with a message giving the size needed; use nw_adjoint then.
 *  - Every GPU that loads the library holds the 64 MiB array until the process exits.
 *  - The first call on a device looks up the array's device address (with that device current) and
 *    caches it; make that first call before any stream capture begins. The cached address belongs to
 *    the device's current context: after cudaDeviceReset (or any teardown of the primary context)
 *    the library must be unloaded and loaded again before this entry point is called.
 *  - All calls share the one array and it keeps the last call's contents; each call clears what it
 *    uses before use, but two calls whose GPU work overlaps (different streams or host threads)
 *    race on it, so serialise them.
 *  - No cudaMalloc, cudaFree or other allocating routine is called.
 */
#define NW_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
int nw_adjoint_grad_c_noalloc(const nw_grid* g, const int32_t* n_abs, const nw_medium* m,
                              const nw_acquisition* a, const nw_time* t, const nw_storage* st,
                              const nw_tuning* tune, const void* c, double dt2,
                              const void* grad_traces, double* grad_c, void* stream);

/*
 * Zero only the ghost cells of `n_fields` consecutive fields (e.g. a freshly allocated history),
 * leaving interior cells untouched: the stencils then read zero outside the grid without a
 * full memset of storage whose interior every step overwrites anyway.
 */
int nw_zero_ghosts(const nw_grid* g, void* fields, int64_t n_fields, void* stream);

/* Number of kernels this library has enqueued since it was loaded (all threads). Host only. */
uint64_t nw_launch_count(void);

/*
 * Batched FWI gradients: many independent 2-D problems (grids of different size, shot counts and
 * step counts, one dtype and stencil order) advanced together, one launch per time step for the
 * whole batch. This has no single counterpart in the reference, whose operators cannot be batched
 * (nefi/solve/batched.py:68-77); each problem's traces and gradient are those nw_forward /
 * nw_adjoint give it alone with the same tuning and snapshots (bitwise).
 *
 * Every problem is an FWI problem (has_source) with checkpointed storage: a ring, a snapshot pool
 * for ceil(n_steps / segment) snapshots, a `segment`-level buffer; `segment` and snap_kind are the
 * same for all problems. Problems must be ordered by non-increasing time.n_steps. The buffers are
 * bound by nw_batch_prepare: later calls use the pointers given there.
 */
typedef struct nw_batch_problem {
  nw_grid grid;
  nw_medium medium;
  nw_acquisition acq;
  nw_time time;
  nw_storage storage;
  void* work;               /* 3 * n_shots fields: the adjoint's levels (PML: 7 * n_shots, with the
                               face cotangents; the PML also needs storage.pml_psi) */
  void* grad_acc;           /* nw_adjoint_groups() fields: c2dt2 * dJ/dc2dt2, as nw_adjoint */
  void* traces;             /* (n_shots, n_rec, n_t): forward output */
  const void* grad_traces;  /* (n_shots, n_rec, n_t): adjoint input */
} nw_batch_problem;

/* Bytes of the device table nw_batch_prepare writes for n_problems problems. */
size_t nw_batch_table_bytes(int32_t n_problems);

/*
 * Validates the batch, builds the per-problem step descriptors and the CTA offsets of the batched
 * launches, and copies them into `table` (nw_batch_table_bytes() bytes of device memory) on
 * `stream`, waiting for the copy. Call once per batch, before any capture of the sweeps.
 */
int nw_batch_prepare(const nw_batch_problem* problems, int32_t n_problems, const nw_tuning* tune,
                     void* table, void* stream);

/*
 * Forward sweep of the whole batch from p^-1 = p^0 = 0: traces of every problem, and the
 * snapshots of every segment start. One kernel per global step over the problems still running
 * (a PML problem's interior box; its layer cells and receivers take launches of their own), plus
 * the snapshot encodes and each problem's final receiver sample. Asynchronous; no host
 * synchronisation, so a caller may capture it in a CUDA graph.
 */
int nw_batch_forward(const nw_batch_problem* problems, int32_t n_problems, const nw_tuning* tune,
                     const void* table, void* stream);

/*
 * Adjoint sweep of the whole batch from each problem's grad_traces: per segment (latest first) the
 * snapshots are decoded and Lap p recomputed for all problems in one kernel per step, then the
 * adjoint steps run for all problems in one kernel per step; grad_acc of every problem is zeroed
 * first and holds the accumulated sums at the end (reduce each with nw_reduce_grad_c).
 * Asynchronous, no host synchronisation.
 */
int nw_batch_adjoint(const nw_batch_problem* problems, int32_t n_problems, const nw_tuning* tune,
                     const void* table, void* stream);

/*
 * Dirichlet time reversal of one trace set (time_reversal(mode="dirichlet"),
 * nefi/physics/wave.py:878-968): starting from rest, the cells `cells` (n_cells distinct ghost-layout
 * offsets, the receivers' nearest cells) hold the traces at reversed time T - n dt, linear in time
 * between samples, at level 0 and after every step n; `traces` is (n_cells, time->n_t) in dtype.
 * The acquisition describes one shot without sources (its receiver tables are not used). The call
 * zeroes st->ring (and st->pml_psi with a PML) and leaves the estimate of p0 in ring level
 * time->n_steps. This has no counterpart in the reference's operators; it replaces the time loop of
 * its `time_reversal`.
 */
int nw_time_reversal(const nw_grid* g, const nw_medium* m, const nw_acquisition* a, const nw_time* t,
                     const nw_storage* st, const nw_tuning* tune, const int64_t* cells, int32_t n_cells,
                     const void* traces, void* stream);

/* Receiver samples of one level (n_shots fields) into traces[:, :, j]. */
int nw_sample(const nw_grid* g, const nw_acquisition* a, int32_t n_t, const void* level,
              int32_t j, void* traces, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Trace misfit: the band-limited relative MSE of FWI (BandLimitedMSE with `lowpass`,
 * nefi/instances/wave_fwi/losses.py:28-86), the sensors' Gaussian response of photoacoustics
 * (gaussian_lowpass, nefi/instances/photoacoustic3d/sensor.py:24-66) and the masked mean of a
 * measurement (nefi/measurement.py:86-91), fused with the adjoint source they feed.
 *
 * Traces are (n_traces, n_t) arrays of dtype, row-major, on the device. A filter is passed as its
 * response: nw_filter_response() writes it on the host (2^log2_len values of dtype, from the
 * reference's own window in float64); copy it to the device once. Every call is asynchronous on
 * `stream`; a state array is one caller-owned device buffer of NW_MISFIT_STATE doubles, and calls
 * that share one state must not overlap on the device.
 * ------------------------------------------------------------------------------------------- */
enum { NW_FILTER_LOWPASS = 0, NW_FILTER_GAUSSIAN = 1 };
#define NW_MISFIT_STATE 2056 /* doubles of a misfit state array */
#define NW_MISFIT_COUNT 2048 /* state slot: the number of observed samples (mask sum) */
#define NW_MISFIT_DEN 2049   /* state slot: masked_mean((W obs)^2) clamped to 1e-30 (1 if not relative) */
#define NW_MISFIT_SCALE 2050 /* state slot: 2 / (count * den), the factor of the adjoint source */
#define NW_MISFIT_SUM 2051   /* state slot: accumulated sum of mask * (W r)^2 */
#define NW_MISFIT_LOSS 2052  /* state slot: the loss, sum / count / den */

typedef struct nw_traces {
  int32_t dtype;           /* NW_F32 or NW_F64 */
  int32_t n_t;             /* samples per trace */
  int64_t n_traces;        /* rows */
  const void* mask;        /* NULL, or observation weights of dtype: one per trace or one per sample */
  int32_t mask_per_sample; /* 0: mask[n_traces]; 1: mask[n_traces * n_t] */
  int32_t log2_len;        /* nw_filter_log2_len(n_t) when a filter is passed (else ignored) */
} nw_traces;

/* Filter length exponent for traces of n_t samples: the smallest k >= 6 with 2^k >= 2 n_t (n_t < 1
 * returns NW_ERR_ARG, a value below 6). Filtered traces are limited to 8192 samples in float32 and
 * 4096 in float64 (the FFT stays in shared memory); nw_filter_response refuses n_t > 8192. */
int nw_filter_log2_len(int32_t n_t);

/*
 * Host: the response of a zero-phase filter on traces of n_t samples at interval dt, written to
 * `out` (host memory, 2^nw_filter_log2_len(n_t) values of dtype). NW_FILTER_LOWPASS: flat to
 * (1 - taper) f, cosine roll-off to 0 at f (`_window`/`lowpass`, losses.py:28-48, FFT length
 * next_fast_len(2 n_t)); NW_FILTER_GAUSSIAN: exp(-(freq / f)^2 / 2) (`gaussian_lowpass`,
 * sensor.py:24-38, FFT length 2 n_t; taper unused).
 */
int nw_filter_response(int32_t kind, int32_t n_t, double dt, double f, double taper, int32_t dtype, void* out);

/* y = the filter `response` applied to every trace of x (lowpass(x) / gaussian_lowpass(x)); the
 * filter is its own adjoint, so the same call maps an output cotangent to the input's. */
int nw_trace_filter(const nw_traces* t, const void* x, const void* response, void* y, void* stream);

/*
 * Once per observed data set: the sample count (mask sum) and, when `relative`, the normaliser
 * masked_mean((W obs)^2) (W = loss_response, or the identity when NULL) go into `state`, with the
 * adjoint-source scale and a zero misfit sum. `t` describes the whole observed set.
 */
int nw_misfit_prepare(const nw_traces* t, const void* obs, const void* loss_response, int32_t relative,
                      double* state, void* stream);

/*
 * One pass over predicted traces (a whole set or a slice of rows of the prepared one):
 *   r = G pred - obs (G = sensor_response, identity when NULL), r_f = W r (W = loss_response),
 *   state[NW_MISFIT_SUM] += sum(mask * r_f^2), state[NW_MISFIT_LOSS] = SUM / COUNT / DEN,
 *   grad = SCALE * G W (mask * r_f)  (= dLoss/dpred; skipped when grad is NULL).
 * One launch plus a one-warp reduction; the partial sums are reduced in a fixed order, so results are
 * bitwise reproducible. Replaces BandLimitedMSE.forward (losses.py:78-86) and its autograd backward.
 */
int nw_misfit(const nw_traces* t, const void* pred, const void* obs, const void* sensor_response,
              const void* loss_response, double* state, void* grad, void* stream);

/*
 * Synchronises `stream`, then returns and clears the device status word that kernels set on a
 * detected failure (a non-finite snapshot block: NW_ERR_NONFINITE). The word is shared by all
 * streams of the current device. NEFI raises OperatorError/SolverError for such failures
 * (nefi/physics/wave.py:561-569, nefi/errors.py:22-27).
 */
int nw_status(void* stream);

/* Message of the calling thread's last error ("" if none). Host only. */
const char* nw_last_error(void);
/* Library ABI version (NW_ABI_VERSION) and the CUDA architecture it was built for (e.g. 1000). */
int nw_abi_version(void);
int nw_built_arch(void);

#ifdef __cplusplus
}
#endif
#endif /* NEFI_WAVE_H */
