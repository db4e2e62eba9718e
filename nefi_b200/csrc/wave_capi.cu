// wave_capi.cu — host drivers and the extern "C" entry points declared in include/nefi_wave.h.
//
// The drivers run whole time loops on the caller's stream (one kernel launch per leapfrog step,
// plus the receiver/adjoint-source kernels), so a forward or adjoint sweep costs one call from
// the host language. No device memory is allocated here: every buffer comes from the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/nefi_wave.h"
#include "aux_kernels.cuh"
#include "kernels.cuh"
#include "misfit.cuh"
#include "pml2d.cuh"
#include "stencil2d.cuh"
#include "stencil3d.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define NW_CUDA(expr)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (expr);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(NW_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));    \
  } while (0)

// Kernels enqueued by this library since load (host-side count, all threads).
std::atomic<unsigned long long> g_launches{0};

#define NW_LAUNCHED()                                                                  \
  do {                                                                                 \
    g_launches.fetch_add(1, std::memory_order_relaxed);                                \
    cudaError_t e_ = cudaGetLastError();                                               \
    if (e_ != cudaSuccess)                                                             \
      return fail(NW_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
  } while (0)

int check_grid(const nw_grid* g) {
  if (!g) return fail(NW_ERR_ARG, "grid is NULL");
  if (g->ndim != 2 && g->ndim != 3) return fail(NW_ERR_UNSUPPORTED, "ndim must be 2 or 3");
  if (g->order != 2 && g->order != 4) return fail(NW_ERR_ARG, "order must be 2 or 4");
  if (g->dtype != NW_F32 && g->dtype != NW_F64) return fail(NW_ERR_ARG, "dtype must be NW_F32 or NW_F64");
  if (g->absorbing < NW_ABS_NONE || g->absorbing > NW_ABS_PML)
    return fail(NW_ERR_UNSUPPORTED, "absorbing kind not built");
  if (g->absorbing == NW_ABS_PML && g->ndim != 2) return fail(NW_ERR_UNSUPPORTED, "the PML is 2-D only");
  for (int a = 0; a < g->ndim; ++a)
    if (g->n[a] < 2) return fail(NW_ERR_ARG, "every padded extent must be >= 2");
  if (g->field_elems >= (1LL << 31)) return fail(NW_ERR_ARG, "a field must hold fewer than 2^31 elements");
  if (g->field_elems <= 0 || g->radius != g->order / 2)
    return fail(NW_ERR_ARG, "grid layout not initialised (call nw_grid_layout)");
  return NW_OK;
}

template <typename T>
nw::KGrid<T> kgrid(const nw_grid* g) {
  nw::KGrid<T> k;
  k.n0 = g->n[0];
  k.n1 = g->n[1];
  k.n2 = g->ndim == 3 ? g->n[2] : 1;
  k.lo0 = g->core_lo[0]; k.lo1 = g->core_lo[1]; k.lo2 = g->ndim == 3 ? g->core_lo[2] : 0;
  k.hi0 = g->core_hi[0]; k.hi1 = g->core_hi[1]; k.hi2 = g->ndim == 3 ? g->core_hi[2] : 1;
  k.s0 = g->stride[0];
  k.s1 = g->stride[1];
  k.origin = g->origin;
  k.field = g->field_elems;
  k.wc = (T)g->w_center;
  k.w1a = (T)g->w1[0]; k.w1b = (T)g->w1[1]; k.w1c = (T)g->w1[2];
  k.w2a = (T)g->w2[0]; k.w2b = (T)g->w2[1]; k.w2c = (T)g->w2[2];
  return k;
}

nw::PadMap padmap(const nw_grid* g, const int32_t* n_abs) {
  nw::PadMap p;
  p.a0 = n_abs[0]; p.a1 = n_abs[1]; p.a2 = g->ndim == 3 ? n_abs[2] : 0;
  p.m0 = g->n[0] - 2 * p.a0; p.m1 = g->n[1] - 2 * p.a1;
  p.m2 = g->ndim == 3 ? g->n[2] - 2 * p.a2 : 1;
  return p;
}

constexpr int kGuard = 32; // zero elements in front of every field (see nw_grid.guard)

// Launch a kernel that may begin while the previous kernel in the stream finishes: the kernel waits
// (griddepcontrol.wait) for that kernel's writes before it touches memory.
template <typename K, typename... Args>
int launch_pdl_b(K kernel, dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  NW_CUDA(cudaLaunchKernelEx(&cfg, kernel, args...));
  NW_LAUNCHED();
  return NW_OK;
}

template <typename T>
int launch_sample(const nw_grid* g, const nw_acquisition* a, int n_t, const T* lvl, int j, T* traces,
                  cudaStream_t s) {
  if (a->n_rec <= 0) return NW_OK;
  dim3 grid((a->n_rec + 127) / 128, a->n_shots);
  const T* w = (const T*)a->rec_weight;
  const int64_t* idx = a->rec_index;
  if (g->ndim == 2)
    return launch_pdl_b(nw::sample_kernel<T, 4>, grid, dim3(128), 0, s, lvl, (long long)g->field_elems, traces, idx, w,
                        (int)a->n_rec, n_t, j);
  return launch_pdl_b(nw::sample_kernel<T, 8>, grid, dim3(128), 0, s, lvl, (long long)g->field_elems, traces, idx, w,
                      (int)a->n_rec, n_t, j);
}

// ---- snapshot pool layout: per snapshot, 2 levels x n_shots fields (with a PML, also the two
// face fields the next step reads: 4 x n_shots) ----------------------------------------------
struct SnapLayout {
  int nblk;             // blocks per field
  size_t vals_bytes;    // 16-bit payload of one snapshot
  size_t scale_bytes;   // scales of one snapshot (delta16: the steps, followed by as many anchors)
  size_t exact_bytes;   // exact copy of one snapshot
  size_t per_snap(int kind) const {
    if (kind == NW_SNAP_EXACT) return exact_bytes;
    const size_t b = vals_bytes + scale_bytes * (kind == NW_SNAP_D16 ? 2 : 1);
    return ((b + 255) / 256) * 256;
  }
};
SnapLayout snap_layout(const nw_grid* g, int n_shots) {
  SnapLayout L;
  const size_t esz = g->dtype == NW_F64 ? 8 : 4;
  L.nblk = (int)((g->field_elems + nw::SNAP_BLOCK - 1) / nw::SNAP_BLOCK);
  const size_t fields = (g->absorbing == NW_ABS_PML ? 4 : 2) * (size_t)n_shots;
  L.vals_bytes = fields * L.nblk * nw::SNAP_BLOCK * 2;
  L.scale_bytes = fields * L.nblk * sizeof(float);
  L.exact_bytes = fields * g->field_elems * esz;
  return L;
}

// Encodes levels (lm1, l0) (each n_shots fields, contiguous) into snapshot j. The 16-bit kinds
// store p^{n0} and the difference p^{n0} - p^{n0-1}, each block-scaled, so the small level
// difference (the discrete time derivative) keeps 16-bit relative precision. With a PML, slots 2
// and 3 hold the two face fields f0, f1 (block-scaled as they are).
template <typename T, int K>
int snap_codec(const nw_grid* g, const SnapLayout& L, int n_shots, char* base, const T* lm1, T* lm1_out,
               const T* l0, T* l0_out, bool encode, cudaStream_t s, const T* const* faces = nullptr,
               T* const* faces_out = nullptr) {
  using H = typename nw::Codec<K>::H;
  float* scales = (float*)(base + L.vals_bytes);
  const size_t half_fields = (size_t)n_shots * L.nblk * nw::SNAP_BLOCK;
  dim3 grid((L.nblk + 8 * nw::SNAP_WARP_BLOCKS - 1) / (8 * nw::SNAP_WARP_BLOCKS), n_shots);
  const int slots = g->absorbing == NW_ABS_PML ? 4 : 2;
  for (int lv = 0; lv < slots; ++lv) {  // slot 0: p^{n0}; slot 1: p^{n0} - p^{n0-1}; 2, 3: faces
    H* v = (H*)base + lv * half_fields;
    float* sc = scales + (size_t)lv * n_shots * L.nblk;
    if (lv >= 2) {
      if (encode)
        nw::snap_encode<T, K><<<grid, 256, 0, s>>>(faces[lv - 2], nullptr, g->field_elems, L.nblk, v, sc);
      else
        nw::snap_decode<T, K><<<grid, 256, 0, s>>>(v, sc, L.nblk, g->field_elems, nullptr, faces_out[lv - 2]);
    } else if (encode) {
      nw::snap_encode<T, K><<<grid, 256, 0, s>>>(l0, lv == 0 ? nullptr : lm1, g->field_elems, L.nblk, v, sc);
    } else {  // p^{n0} first, then p^{n0-1} = p^{n0} - difference
      nw::snap_decode<T, K><<<grid, 256, 0, s>>>(v, sc, L.nblk, g->field_elems, lv == 0 ? nullptr : l0_out,
                                                 lv == 0 ? l0_out : lm1_out);
    }
    NW_LAUNCHED();
  }
  return NW_OK;
}

// delta16 snapshots (nw::snap_encode_d16): both pressure slots in one launch, and the face slots
// in the same launch with a PML; decoding writes p^{n0} and p^{n0-1} from one pass over the slots.
template <typename T>
int snap_codec_d16(const nw_grid* g, const SnapLayout& L, int n_shots, char* base, const T* lm1, T* lm1_out,
                   const T* l0, T* l0_out, bool encode, cudaStream_t s, const T* const* faces = nullptr,
                   T* const* faces_out = nullptr) {
  short* vals = (short*)base;
  float* steps = (float*)(base + L.vals_bytes);
  float* anchors = (float*)(base + L.vals_bytes + L.scale_bytes);
  const int slots = g->absorbing == NW_ABS_PML ? 4 : 2;
  if (g->field_elems % nw::SNAP_BLOCK != 0 || g->origin % nw::SNAP_BLOCK != 0)
    return fail(NW_ERR_UNSUPPORTED, "delta16 snapshots need fields and rows on multiples of 32 elements");
  constexpr int blk = nw::D16Cta<T>::BLK;
  const unsigned gx = (unsigned)((L.nblk + blk - 1) / blk);
  if (encode) {
    nw::snap_encode_d16<T><<<dim3(gx, n_shots, slots), 256, 0, s>>>(
        lm1, l0, slots == 4 ? faces[0] : nullptr, slots == 4 ? faces[1] : nullptr, g->field_elems, L.nblk, vals,
        steps, anchors);
  } else {
    nw::snap_decode_d16<T><<<dim3(gx, n_shots, slots / 2), 256, 0, s>>>(
        vals, steps, anchors, L.nblk, g->field_elems, kgrid<T>(g), g->ndim, lm1_out, l0_out,
        slots == 4 ? faces_out[0] : nullptr, slots == 4 ? faces_out[1] : nullptr);
  }
  NW_LAUNCHED();
  return NW_OK;
}

// The two PML face fields that step n reads (parity n % 2 of the double-buffered levels).
template <typename T>
void pml_faces(T* psi, long long level_elems, int n, T* out[2]) {
  for (int ax = 0; ax < 2; ++ax) out[ax] = psi + (long long)(2 * ax + n % 2) * level_elems;
}

// Snapshot j of the levels (lm1, l0) and, with a PML, of the face fields `faces` (NULL otherwise).
template <typename T>
int snap_store(const nw_grid* g, const nw_storage* st, int n_shots, const T* lm1, const T* l0, int j,
               cudaStream_t s, T* const* faces = nullptr) {
  SnapLayout L = snap_layout(g, n_shots);
  char* base = (char*)st->snap + (size_t)j * L.per_snap(st->snap_kind);
  const size_t lvl_bytes = (size_t)n_shots * g->field_elems * sizeof(T);
  const T* const* fc = (const T* const*)faces;
  switch (st->snap_kind) {
    case NW_SNAP_EXACT:
      NW_CUDA(cudaMemcpyAsync(base, lm1, lvl_bytes, cudaMemcpyDeviceToDevice, s));
      NW_CUDA(cudaMemcpyAsync(base + lvl_bytes, l0, lvl_bytes, cudaMemcpyDeviceToDevice, s));
      if (faces)
        for (int f = 0; f < 2; ++f)
          NW_CUDA(cudaMemcpyAsync(base + (2 + f) * lvl_bytes, faces[f], lvl_bytes, cudaMemcpyDeviceToDevice, s));
      return NW_OK;
    case NW_SNAP_F16: return snap_codec<T, nw::CODEC_F16>(g, L, n_shots, base, lm1, nullptr, l0, nullptr, true, s, fc);
    case NW_SNAP_BF16: return snap_codec<T, nw::CODEC_BF16>(g, L, n_shots, base, lm1, nullptr, l0, nullptr, true, s, fc);
    case NW_SNAP_I16: return snap_codec<T, nw::CODEC_I16>(g, L, n_shots, base, lm1, nullptr, l0, nullptr, true, s, fc);
    case NW_SNAP_D16: return snap_codec_d16<T>(g, L, n_shots, base, lm1, nullptr, l0, nullptr, true, s, fc);
  }
  return fail(NW_ERR_ARG, "unknown snapshot kind");
}

template <typename T>
int snap_load(const nw_grid* g, const nw_storage* st, int n_shots, int j, T* lm1, T* l0,
              cudaStream_t s, T* const* faces = nullptr) {
  SnapLayout L = snap_layout(g, n_shots);
  char* base = (char*)st->snap + (size_t)j * L.per_snap(st->snap_kind);
  const size_t lvl_bytes = (size_t)n_shots * g->field_elems * sizeof(T);
  switch (st->snap_kind) {
    case NW_SNAP_EXACT:
      NW_CUDA(cudaMemcpyAsync(lm1, base, lvl_bytes, cudaMemcpyDeviceToDevice, s));
      NW_CUDA(cudaMemcpyAsync(l0, base + lvl_bytes, lvl_bytes, cudaMemcpyDeviceToDevice, s));
      if (faces)
        for (int f = 0; f < 2; ++f)
          NW_CUDA(cudaMemcpyAsync(faces[f], base + (2 + f) * lvl_bytes, lvl_bytes, cudaMemcpyDeviceToDevice, s));
      return NW_OK;
    case NW_SNAP_F16:
      return snap_codec<T, nw::CODEC_F16>(g, L, n_shots, base, nullptr, lm1, nullptr, l0, false, s, nullptr, faces);
    case NW_SNAP_BF16:
      return snap_codec<T, nw::CODEC_BF16>(g, L, n_shots, base, nullptr, lm1, nullptr, l0, false, s, nullptr, faces);
    case NW_SNAP_I16:
      return snap_codec<T, nw::CODEC_I16>(g, L, n_shots, base, nullptr, lm1, nullptr, l0, false, s, nullptr, faces);
    case NW_SNAP_D16:
      return snap_codec_d16<T>(g, L, n_shots, base, nullptr, lm1, nullptr, l0, false, s, nullptr, faces);
  }
  return fail(NW_ERR_ARG, "unknown snapshot kind");
}

// ---- launch shapes ------------------------------------------------------------------------
struct TileCfg {  // one 2-D step kernel's tile: 8*rx rows by 32*vz columns, spc shots per CTA
  int vz, rx, spc;
  int depth = 1;   // forward steps per launch; with 2 the tile is the core of that shape (fwd2t)
  int r = 0, hl = 0;  // stencil radius and halo columns (16 bytes of elements) of the grid
  int tx() const { return 8 * rx - (depth == 2 ? 2 * r : 0); }
  int tz() const { return 32 * vz - (depth == 2 ? 2 * hl : 0); }
  int tiles_z(const nw_grid* g) const { return (g->n[1] + tz() - 1) / tz(); }
  int groups(int n_shots) const { return (n_shots + spc - 1) / spc; }
  dim3 grid(const nw_grid* g, int n_shots) const {
    return dim3(tiles_z(g), (g->n[0] + tx() - 1) / tx(), groups(n_shots));
  }
};
struct Tune {
  TileCfg fwd, adj;
};

int check_tile(const nw_grid* g, const TileCfg& c, const char* which) {
  const std::string w(which);
  if (g->dtype == NW_F32 && c.vz != 2 && c.vz != 4) return fail(NW_ERR_ARG, "tuning." + w + "vz must be 2 or 4 for float32");
  if (g->dtype == NW_F64 && c.vz != 2) return fail(NW_ERR_ARG, "tuning." + w + "vz must be 2 for float64");
  if (c.rx != 2 && c.rx != 4 && c.rx != 8) return fail(NW_ERR_ARG, "tuning." + w + "rx must be 2, 4 or 8");
  if (c.spc < 1) return fail(NW_ERR_ARG, "tuning." + w + "shots_per_cta must be >= 1");
  return NW_OK;
}

int resolve_tune(const nw_grid* g, const nw_tuning* t, Tune* out) {
  Tune r;
  // defaults: the best forward and adjoint times of a sweep on a 552^2 x 16-shot grid
  r.fwd.vz = (t && t->vz) ? t->vz : (g->dtype == NW_F32 ? 4 : 2);
  r.fwd.rx = (t && t->rx) ? t->rx : 2;
  r.fwd.spc = (t && t->shots_per_cta) ? t->shots_per_cta : 2;
  r.adj.vz = (t && t->adj_vz) ? t->adj_vz : 2;
  r.adj.rx = (t && t->adj_rx) ? t->adj_rx : 2;
  r.adj.spc = (t && t->adj_shots_per_cta) ? t->adj_shots_per_cta : 4;
  int rc = check_tile(g, r.fwd, "");
  if (rc) return rc;
  rc = check_tile(g, r.adj, "adj_");
  if (rc) return rc;
  if (g->ndim == 3) r.fwd.spc = r.adj.spc = 1;
  // two forward steps per launch: 2-D grids without a PML (whose steps run a layer kernel beside the box)
  r.fwd.depth = (t && t->depth == 2 && g->ndim == 2 && g->absorbing != NW_ABS_PML) ? 2 : 1;
  if (t && (t->depth < 0 || t->depth > 2)) return fail(NW_ERR_ARG, "tuning.depth must be 0, 1 or 2");
  r.fwd.r = r.adj.r = g->radius;
  r.fwd.hl = r.adj.hl = g->dtype == NW_F64 ? 2 : 4;
  *out = r;
  return NW_OK;
}

// Accumulator fields the adjoint fills: one per shot in 3-D and with a PML, one per adjoint shot
// group for the tiled 2-D steps.
int n_acc_fields(const nw_grid* g, const Tune& t, int n_shots) {
  return (g->ndim == 3 || g->absorbing == NW_ABS_PML) ? n_shots : t.adj.groups(n_shots);
}
// Levels of nw_adjoint's work buffer: q^{n..n+2}, and with a PML the face cotangents.
int work_levels(const nw_grid* g) { return g->absorbing == NW_ABS_PML ? 7 : 3; }

// Dynamic shared memory: fwd2d stages C, A, B and the ring of p^n halo tiles; adj2d stages C, A, B, the
// accumulator tile, the ring of (q^{n+1} halo, q^{n+2} core, Lap p^n core) tiles and one shot's
// injected cotangents.
template <typename T, int R, int VZ, int RX, bool ADJ>
constexpr size_t step2_smem() {
  using S = nw::Tile2Shape<T, VZ, RX, R>;
  return (ADJ ? 6 * S::QS + S::NSA * (S::PS + 2 * S::QS) : 3 * S::QS + S::NS * S::PS) * sizeof(T);
}
// fwd2t: C, A, B over the extended tile, the shared p^{n+1} tile and the ring of p^n halo tiles.
template <typename T, int R, int VZ, int RX>
constexpr size_t step2t_smem() {
  using S = nw::Tile2Shape<T, VZ, RX, R>;
  return (3 * S::QS + (nw::Tile2T<T, VZ, RX, R>::NS + 1) * S::PS) * sizeof(T);
}
constexpr size_t kMaxSmem = 227 * 1024;  // opt-in shared memory per CTA on sm_100a

// Opt a kernel into more than 48 KB of dynamic shared memory (once per instantiation).
template <typename K>
int allow_smem(K kernel, size_t bytes, bool* done) {
  if (*done || bytes <= 48 * 1024) return NW_OK;
  NW_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  *done = true;
  return NW_OK;
}

// Launch a step kernel that may begin while the previous kernel in the stream finishes: the
// kernel waits (griddepcontrol.wait) for that kernel's writes before it reads any field.
template <typename K, typename... Args>
int launch_pdl(K kernel, dim3 grid, size_t smem, cudaStream_t s, Args... args) {
  return launch_pdl_b(kernel, grid, dim3(256, 1, 1), smem, s, args...);
}

nw::TileTables tile_tables(const nw_grid* g, const nw_acquisition* a, const TileCfg& c) {
  nw::TileTables tt;
  tt.tiles_z = c.tiles_z(g);
  tt.rec_ptr = a->tile_rec_ptr;
  tt.rec_list = a->tile_rec_list;
  tt.rec_corner = a->rec_corner;
  tt.cell_ptr = a->tile_cell_ptr;
  tt.cell_local = a->tile_cell_local;
  tt.cell_gid = a->tile_cell_gid;
  tt.gcell_ptr = a->cell_ptr;
  tt.gcell_rec = a->cell_rec;
  return tt;
}

// A descriptor without a sub-box (x_end = 0) covers the whole grid.
template <typename T>
nw::Tiled2<T> whole_grid(const nw::KGrid<T>& kg, nw::Tiled2<T> st) {
  if (st.x_end == 0) {
    st.tx_off = st.tz_off = 0;
    st.x_end = kg.n0;
    st.z_end = kg.n1;
  }
  return st;
}

template <typename T, int R, int VZ, int RX, bool AB>
int launch_fwd2_v(const nw::KGrid<T>& kg, const nw::Tiled2<T>& st, dim3 grid, cudaStream_t s) {
  constexpr size_t smem = step2_smem<T, R, VZ, RX, false>();
  if (smem > kMaxSmem) return fail(NW_ERR_ARG, "tile too large for shared memory (lower tuning rx or vz)");
  static bool done = false;
  int rc = allow_smem(nw::fwd2d<T, R, VZ, RX, AB>, smem, &done);
  if (rc) return rc;
  return launch_pdl(nw::fwd2d<T, R, VZ, RX, AB>, grid, smem, s, kg, whole_grid(kg, st));
}
template <typename T, int R, int VZ, int RX, bool AB>
int launch_fwd2t_v(const nw::KGrid<T>& kg, const nw::Tiled2<T>& st, dim3 grid, cudaStream_t s) {
  constexpr size_t smem = step2t_smem<T, R, VZ, RX>();
  if constexpr (smem > kMaxSmem) {
    return fail(NW_ERR_ARG, "two-step tile too large for shared memory (lower tuning rx or vz)");
  } else {
    static bool done = false;
    int rc = allow_smem(nw::fwd2t<T, R, VZ, RX, AB>, smem, &done);
    if (rc) return rc;
    return launch_pdl(nw::fwd2t<T, R, VZ, RX, AB>, grid, smem, s, kg, st);
  }
}
template <typename T, int R, int VZ, int RX, bool AB>
int launch_adj2_v(const nw::KGrid<T>& kg, const nw::Tiled2<T>& st, dim3 grid, cudaStream_t s) {
  constexpr size_t smem = step2_smem<T, R, VZ, RX, true>();
  if (smem > kMaxSmem) return fail(NW_ERR_ARG, "tile too large for shared memory (lower tuning adj_rx or adj_vz)");
  static bool done = false;
  int rc = allow_smem(nw::adj2d<T, R, VZ, RX, AB>, smem, &done);
  if (rc) return rc;
  return launch_pdl(nw::adj2d<T, R, VZ, RX, AB>, grid, smem, s, kg, whole_grid(kg, st));
}

// 3-D step: forward (ADJ = false) or adjoint, plane-marching tiles of 8 x 64 (y, z) cells over chunks
// of kXChunk planes (16-row tiles of 16 warps measured 7 % slower on the 256^3 photoacoustic gradient).
constexpr int kXChunk = 32;
template <typename T, int R, bool ADJ>
int launch_step3_r(const nw_grid* g, const nw::KGrid<T>& kg, const nw::Step3<T>& st, int n_shots, cudaStream_t s) {
  using S = nw::Tile3Shape<T, 2, R>;
  const int tz = (g->n[2] + S::TZ - 1) / S::TZ, ty = (g->n[1] + S::TY - 1) / S::TY;
  if ((long long)tz * ty * n_shots > INT_MAX) return fail(NW_ERR_UNSUPPORTED, "3-D grid: too many tiles x shots");
  const dim3 grid((unsigned)((long long)tz * ty * n_shots), (g->n[0] + kXChunk - 1) / kXChunk);  // shot fastest
  constexpr size_t smem = (size_t)S::NSP * S::PS * sizeof(T);
  static_assert(smem <= kMaxSmem, "plane ring above the shared-memory limit");
  static bool done = false;
  int rc = allow_smem(nw::step3t<T, R, 2, ADJ>, smem, &done);
  if (rc) return rc;
  return launch_pdl_b(nw::step3t<T, R, 2, ADJ>, grid, dim3(S::NT), smem, s, kg, st, kXChunk, n_shots);
}
template <typename T, bool ADJ>
int launch_step3(const nw_grid* g, const nw::KGrid<T>& kg, const nw::Step3<T>& st, bool ab, int n_shots,
                 cudaStream_t s) {
  (void)ab;  // the kernel reads A/B in layer cells when the medium has them
  return g->radius == 1 ? launch_step3_r<T, 1, ADJ>(g, kg, st, n_shots, s) : launch_step3_r<T, 2, ADJ>(g, kg, st, n_shots, s);
}

// Runtime (radius, vz, rx, absorbing) -> template instantiation.
#define NW_DISPATCH2(FN, T, TU, ...)                                                                   \
  [&]() -> int {                                                                                   \
    const int r_ = g->radius;                                                                      \
    const bool ab_ = m->coef_a != nullptr;                                                         \
    if constexpr (sizeof(T) == 4) {                                                                \
      if (TU.vz == 4) {                                                                             \
        if (r_ == 2) {                                                                             \
          if (TU.rx == 2) return ab_ ? FN<T, 2, 4, 2, true>(__VA_ARGS__) : FN<T, 2, 4, 2, false>(__VA_ARGS__); \
          if (TU.rx == 4) return ab_ ? FN<T, 2, 4, 4, true>(__VA_ARGS__) : FN<T, 2, 4, 4, false>(__VA_ARGS__); \
          return ab_ ? FN<T, 2, 4, 8, true>(__VA_ARGS__) : FN<T, 2, 4, 8, false>(__VA_ARGS__);     \
        }                                                                                          \
        if (TU.rx == 2) return ab_ ? FN<T, 1, 4, 2, true>(__VA_ARGS__) : FN<T, 1, 4, 2, false>(__VA_ARGS__); \
        if (TU.rx == 4) return ab_ ? FN<T, 1, 4, 4, true>(__VA_ARGS__) : FN<T, 1, 4, 4, false>(__VA_ARGS__); \
        return ab_ ? FN<T, 1, 4, 8, true>(__VA_ARGS__) : FN<T, 1, 4, 8, false>(__VA_ARGS__);       \
      }                                                                                            \
    }                                                                                              \
    if (r_ == 2) {                                                                                 \
      if (TU.rx == 2) return ab_ ? FN<T, 2, 2, 2, true>(__VA_ARGS__) : FN<T, 2, 2, 2, false>(__VA_ARGS__); \
      if (TU.rx == 4) return ab_ ? FN<T, 2, 2, 4, true>(__VA_ARGS__) : FN<T, 2, 2, 4, false>(__VA_ARGS__); \
      return ab_ ? FN<T, 2, 2, 8, true>(__VA_ARGS__) : FN<T, 2, 2, 8, false>(__VA_ARGS__);         \
    }                                                                                              \
    if (TU.rx == 2) return ab_ ? FN<T, 1, 2, 2, true>(__VA_ARGS__) : FN<T, 1, 2, 2, false>(__VA_ARGS__); \
    if (TU.rx == 4) return ab_ ? FN<T, 1, 2, 4, true>(__VA_ARGS__) : FN<T, 1, 2, 4, false>(__VA_ARGS__); \
    return ab_ ? FN<T, 1, 2, 8, true>(__VA_ARGS__) : FN<T, 1, 2, 8, false>(__VA_ARGS__);           \
  }()

// ---- forward driver ---------------------------------------------------------------------
// The PML coefficients of a medium into a step descriptor.
template <typename T>
void pml_medium(const nw_medium* m, nw::PmlStep<T>& st) {
  st.C = (const T*)m->c2dt2;
  st.A = (const T*)m->coef_a;
  st.B = (const T*)m->coef_b;
  st.ZZ = (const T*)m->pml_zz;
  for (int ax = 0; ax < 2; ++ax) {
    st.alpha[ax] = (const T*)m->pml_alpha[ax];
    st.beta[ax] = (const T*)m->pml_beta[ax];
  }
  st.hx2 = (T)m->pml_half_inv_h[0];
  st.hz2 = (T)m->pml_half_inv_h[1];
  st.cx0 = m->pml_core[0];
  st.cx1 = m->pml_core[1];
  st.cz0 = m->pml_core[2];
  st.cz1 = m->pml_core[3];
}

template <typename T, bool ADJ>
int launch_pml(const nw_grid* g, const nw::KGrid<T>& kg, const nw::PmlStep<T>& st, int n_shots, cudaStream_t s) {
  const long long vecs =
      nw::pml_layer_vectors(g->n[0], g->n[1], st.kx0, st.kx1, st.kz0, st.kz1, 16 / (int)sizeof(T));
  if (vecs <= 0 && !st.traces) return NW_OK;
  // a thread per 16-byte vector of layer cells and shot, and with st.traces the CTAs that take the
  // receiver samples
  const int rec_ctas = st.traces ? (st.n_rec + nw::PML_THREADS - 1) / nw::PML_THREADS : 0;
  const dim3 grid((unsigned)((vecs + nw::PML_THREADS - 1) / nw::PML_THREADS + rec_ctas), n_shots),
      block(nw::PML_THREADS);
  if (g->radius == 1) return launch_pdl_b(nw::pml2d_step<T, 1, ADJ>, grid, block, 0, s, kg, st);
  return launch_pdl_b(nw::pml2d_step<T, 2, ADJ>, grid, block, 0, s, kg, st);
}

// A second stream of the calling thread on the current device, with a fork and a join event: a PML
// step runs its layer kernel there beside the interior box's tiled kernel (the two write disjoint
// cells and read the same levels), forked from and joined back into the caller's stream, so stream
// order (and a CUDA-graph capture of the caller's stream) is kept. Created at first use, kept until
// the process exits.
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
int side_stream(SideStream** out) {
  thread_local SideStream per_device[64];
  int dev = 0;
  NW_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(NW_ERR_UNSUPPORTED, "device index above 63");
  SideStream& r = per_device[dev];
  if (!r.s) {  // created in relaxed capture mode, so a first call inside a stream capture is safe too
    cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
    NW_CUDA(cudaThreadExchangeStreamCaptureMode(&mode));
    const cudaError_t e0 = cudaStreamCreateWithFlags(&r.s, cudaStreamNonBlocking);
    const cudaError_t e1 = e0 ? e0 : cudaEventCreateWithFlags(&r.fork, cudaEventDisableTiming);
    const cudaError_t e2 = e1 ? e1 : cudaEventCreateWithFlags(&r.join, cudaEventDisableTiming);
    NW_CUDA(cudaThreadExchangeStreamCaptureMode(&mode));
    if (e2 != cudaSuccess) {
      r.s = nullptr;
      return fail(NW_ERR_CUDA, std::string("side stream: ") + cudaGetErrorString(e2));
    }
  }
  *out = &r;
  return NW_OK;
}

// side(t) on the calling thread's second stream beside main(s), both ordered after the work already
// in s and joined back into it (with no side work, main(s) alone). Once the side stream is forked it
// is joined back on every path, errors included, so a capture of s never ends with it still forked;
// the first error is the one returned.
template <typename FS, typename FM>
int fork_join(cudaStream_t s, bool with_side, FS side, FM main) {
  if (!with_side) return main(s);
  SideStream* ss = nullptr;
  int rc = side_stream(&ss);
  if (rc) return rc;
  NW_CUDA(cudaEventRecord(ss->fork, s));
  NW_CUDA(cudaStreamWaitEvent(ss->s, ss->fork, 0));
  rc = side(ss->s);
  const cudaError_t ej = cudaEventRecord(ss->join, ss->s);
  if (rc == NW_OK && ej == cudaSuccess) rc = main(s);
  const cudaError_t ew = ej == cudaSuccess ? cudaStreamWaitEvent(s, ss->join, 0) : ej;
  if (rc) return rc;
  if (ew != cudaSuccess) return fail(NW_ERR_CUDA, std::string("side stream join: ") + cudaGetErrorString(ew));
  return NW_OK;
}

// The PML's interior box that the tiled kernels step (nw_medium.pml_core with its first column rounded
// up to a 16-byte chunk), recorded in st.k*; left empty when the core box is missing or smaller than
// one tile of `c`. Returns an error for a core box outside the grid.
template <typename T>
int pml_tiled_box(const nw_grid* g, const nw_medium* m, const TileCfg& c, nw::PmlStep<T>& st) {
  constexpr int epc = 16 / (int)sizeof(T);
  int x0 = m->pml_core[0], x1 = m->pml_core[1], z0 = m->pml_core[2], z1 = m->pml_core[3];
  if (x0 < 0 || z0 < 0 || x1 < x0 || z1 < z0 || x1 > g->n[0] || z1 > g->n[1])
    return fail(NW_ERR_ARG, "medium.pml_core lies outside the grid");
  z0 = (z0 + epc - 1) / epc * epc;
  if (x1 - x0 < c.tx() || z1 - z0 < c.tz()) x0 = x1 = z0 = z1 = 0;
  st.kx0 = x0;
  st.kx1 = x1;
  st.kz0 = z0;
  st.kz1 = z1;
  return NW_OK;
}

// Tiled-kernel descriptor of that box: tiles from its corner, stores below its end.
template <typename T>
dim3 box_tiles(const nw::PmlStep<T>& st, const TileCfg& c, int n_shots, nw::Tiled2<T>& tb) {
  tb.tx_off = st.kx0;
  tb.tz_off = st.kz0;
  tb.x_end = st.kx1;
  tb.z_end = st.kz1;
  tb.n_shots = n_shots;
  tb.shots_per_cta = c.spc;
  tb.tt.tiles_z = (st.kz1 - st.kz0 + c.tz() - 1) / c.tz();
  return dim3(tb.tt.tiles_z, (st.kx1 - st.kx0 + c.tx() - 1) / c.tx(), c.groups(n_shots));
}

// The receiver cotangents of step n's touched layer cells, added by the PML layer launch itself.
template <typename T>
void layer_inject(const nw_acquisition* a, const T* gtr, int n_t, int j, nw::PmlStep<T>& ps) {
  if (a->n_layer_cells <= 0) return;
  ps.gtr = gtr;
  ps.n_rec = (int)a->n_rec;
  ps.n_t = n_t;
  ps.j = j;
  ps.lc_off = a->layer_cell_index;
  ps.lc_gid = a->layer_cell_gid;
  ps.n_lc = a->n_layer_cells;
  ps.gc_ptr = a->cell_ptr;
  ps.gc_rec = a->cell_rec;
  ps.gc_w = (const T*)a->cell_weight;
}

// Whether the PML's interior box (tiled by `c` from its corner (kx0, kz0), tiles_z tiles along z)
// adds the receiver cotangents in its own adjoint launch: the acquisition's adjoint tile tables were
// built for exactly these tiles, and the touched cells outside the box are listed for the layer's
// launch.
inline bool box_injects(const nw_acquisition* a, const TileCfg& c, int kx0, int kz0, int tiles_z) {
  return a->n_cells > 0 && a->adj_tables_box && a->tile_cell_ptr &&
         (a->n_layer_cells == 0 || (a->layer_cell_index && a->layer_cell_gid)) && a->adj_box_corner[0] == kx0 &&
         a->adj_box_corner[1] == kz0 && a->adj_tiles_z == tiles_z && a->adj_tile_rows == c.tx() &&
         a->adj_tile_cols == c.tz();
}

template <typename T>
struct Ring {  // time level n (n >= -1) of the pressure field: three (or four) rotating levels
  T* base;
  long long level_elems;
  int levels = 3;
  T* at(int n) const { return base + (long long)((n + 1) % levels) * level_elems; }
};
int ring_levels(const nw_storage* st) { return st->ring_levels == 4 ? 4 : 3; }

// Two forward steps n, n+1 for all shots in one launch (fwd2t): 2-D without a PML, tuning depth 2,
// a ring of four levels. Receivers of levels n and n+1 on record steps; Lap p^n and Lap p^{n+1} into
// lap0 / lap1 when given. two = false: the step n alone with the same tiles.
template <typename T>
int forward_pair(const nw_grid* g, const nw::KGrid<T>& kg, const nw_medium* m, const nw_acquisition* a,
                 const nw_time* t, const Tune& tu, const Ring<T>& L, int n, bool two, T* traces, T* lap0,
                 T* lap1, cudaStream_t s) {
  if (two && L.levels != 4) return fail(NW_ERR_ARG, "two steps per launch need a ring of four levels");
  nw::Tiled2<T> st = {};
  st.prev = L.at(n - 1);
  st.cur = L.at(n);
  st.next = L.at(n + 1);
  st.next2 = two ? L.at(n + 2) : nullptr;
  st.lap_out = lap0;
  st.lap_out1 = two ? lap1 : nullptr;
  st.two = two ? 1 : 0;
  st.C = (const T*)m->c2dt2;
  st.A = (const T*)m->coef_a;
  st.B = (const T*)m->coef_b;
  st.b_one = (n == 0 && t->first_b_one) ? 1 : 0;
  st.prev_ready = 0;  // the previous launch may have written p^{n-1} as its second step
  st.src_corner = a->has_source ? a->src_corner : nullptr;
  st.src_w = (const T*)a->src_weight;
  st.wavelet = (const T*)a->wavelet;
  st.n = n;
  st.n_shots = a->n_shots;
  st.shots_per_cta = tu.fwd.spc;
  const bool rec0 = traces && a->n_rec > 0 && n % t->substeps == 0;
  const bool rec1 = two && traces && a->n_rec > 0 && (n + 1) % t->substeps == 0;
  st.traces = rec0 ? traces : nullptr;
  st.traces1 = rec1 ? traces : nullptr;
  st.j = n / t->substeps;
  st.j1 = (n + 1) / t->substeps;
  st.rec_w = (const T*)a->rec_weight;
  st.n_rec = a->n_rec;
  st.n_t = t->n_t;
  st.tt = tile_tables(g, a, tu.fwd);
  st.x_end = g->n[0];
  st.z_end = g->n[1];
  return NW_DISPATCH2(launch_fwd2t_v, T, tu.fwd, kg, st, tu.fwd.grid(g, a->n_shots), s);
}


// One forward step n for all shots (traces != NULL: also sample level n if it is a record step;
// lap_out != NULL: also store Lap p^n there, the factor of the step's velocity gradient term).
template <typename T>
int forward_step(const nw_grid* g, const nw::KGrid<T>& kg, const nw_medium* m, const nw_acquisition* a,
                 const nw_time* t, const Tune& tu, const Ring<T>& L, int n, T* traces, T* lap_out,
                 cudaStream_t s, T* psi = nullptr, bool prev_ready = false) {
  const bool rec = traces && a->n_rec > 0 && (n % t->substeps) == 0;
  if (g->absorbing == NW_ABS_PML) {  // 2-D with the reference's PML: psi levels 2*axis + parity
    const long long LE = (long long)a->n_shots * g->field_elems;
    nw::PmlStep<T> st = {};
    if (rec) {  // the layer kernel's launch also takes the receiver samples of p^n
      st.traces = traces;
      st.rec_idx = a->rec_index;
      st.rec_w = (const T*)a->rec_weight;
      st.n_rec = (int)a->n_rec;
      st.n_t = t->n_t;
      st.j = n / t->substeps;
    }
    st.prev = L.at(n - 1);
    st.cur = L.at(n);
    st.next = L.at(n + 1);
    pml_medium(m, st);
    for (int ax = 0; ax < 2; ++ax) {
      st.f_old[ax] = psi + (long long)(2 * ax + n % 2) * LE;
      st.f_new[ax] = psi + (long long)(2 * ax + (n + 1) % 2) * LE;
    }
    st.src_corner = a->has_source ? a->src_corner : nullptr;
    st.src_w = (const T*)a->src_weight;
    st.wavelet = (const T*)a->wavelet;
    st.n = n;
    st.lap_out = lap_out;
    int rc = pml_tiled_box<T>(g, m, tu.fwd, st);
    if (rc) return rc;
    if (st.kx1 == st.kx0) return launch_pml<T, false>(g, kg, st, a->n_shots, s);  // no interior box
    nw::Tiled2<T> tb = {};  // the interior box: the plain step (A = B = 1 and no PML term there)
    tb.prev = st.prev;
    tb.cur = st.cur;
    tb.next = st.next;
    tb.lap_out = lap_out;
    tb.C = (const T*)m->c2dt2;
    tb.A = (const T*)m->coef_a;
    tb.B = (const T*)m->coef_b;
    tb.src_corner = st.src_corner;
    tb.src_w = st.src_w;
    tb.wavelet = st.wavelet;
    tb.n = n;
    const dim3 grid = box_tiles<T>(st, tu.fwd, a->n_shots, tb);
    // the layer on the side stream beside the box; the step ends when both halves have
    return fork_join(
        s, true, [&](cudaStream_t t) { return launch_pml<T, false>(g, kg, st, a->n_shots, t); },
        [&](cudaStream_t t) { return NW_DISPATCH2(launch_fwd2_v, T, tu.fwd, kg, tb, grid, t); });
  }
  if (g->ndim == 2 && tu.fwd.depth == 2)  // the two-step kernel's tiles, one step
    return forward_pair<T>(g, kg, m, a, t, tu, L, n, false, traces, lap_out, nullptr, s);
  if (g->ndim == 2) {
    nw::Tiled2<T> st = {};
    st.prev = L.at(n - 1);
    st.cur = L.at(n);
    st.next = L.at(n + 1);
    st.lap_out = lap_out;
    st.C = (const T*)m->c2dt2;
    st.A = (const T*)m->coef_a;
    st.B = (const T*)m->coef_b;
    st.b_one = (n == 0 && t->first_b_one) ? 1 : 0;
    st.prev_ready = prev_ready ? 1 : 0;
    st.src_corner = a->has_source ? a->src_corner : nullptr;
    st.src_w = (const T*)a->src_weight;
    st.wavelet = (const T*)a->wavelet;
    st.n = n;
    st.n_shots = a->n_shots;
    st.shots_per_cta = tu.fwd.spc;
    st.traces = rec ? traces : nullptr;
    st.rec_w = (const T*)a->rec_weight;
    st.n_rec = a->n_rec;
    st.n_t = t->n_t;
    st.j = n / t->substeps;
    st.tt = tile_tables(g, a, tu.fwd);
    return NW_DISPATCH2(launch_fwd2_v, T, tu.fwd, kg, st, tu.fwd.grid(g, a->n_shots), s);
  }
  nw::Step3<T> st = {};
  st.prev = L.at(n - 1);
  st.cur = L.at(n);
  st.next = L.at(n + 1);
  st.lap_out = lap_out;
  st.C = (const T*)m->c2dt2;
  st.A = (const T*)m->coef_a;
  st.B = (const T*)m->coef_b;
  st.b_one = (n == 0 && t->first_b_one) ? 1 : 0;
  st.src_corner = a->has_source ? a->src_corner : nullptr;
  st.src_w = (const T*)a->src_weight;
  st.wavelet = (const T*)a->wavelet;
  st.n = n;
  st.traces = rec ? traces : nullptr;
  st.rec_idx = a->rec_index;
  st.rec_w = (const T*)a->rec_weight;
  st.n_rec = a->n_rec;
  st.n_t = t->n_t;
  st.j = n / t->substeps;
  return launch_step3<T, false>(g, kg, st, m->coef_a != nullptr, a->n_shots, s);
}

template <typename T>
int forward_impl(const nw_grid* g, const nw_medium* m, const nw_acquisition* a, const nw_time* t,
                 const nw_storage* st, const Tune& tu, int n_begin, int n_end, T* traces, cudaStream_t s) {
  const long long LE = (long long)a->n_shots * g->field_elems;
  if (!st->ring) return fail(NW_ERR_ARG, "storage needs a ring buffer");
  Ring<T> L;
  L.base = (T*)st->ring;
  L.level_elems = LE;
  L.levels = ring_levels(st);
  const bool ckpt = !st->history && st->snap;
  if (ckpt && st->segment < 1) return fail(NW_ERR_ARG, "segment must be >= 1");
  const bool pml = g->absorbing == NW_ABS_PML;
  if (pml && !st->pml_psi) return fail(NW_ERR_ARG, "a PML run needs storage.pml_psi");
  const nw::KGrid<T> kg = kgrid<T>(g);
  // a segment start's snapshot slot (segment j -> slot j, or the binomial schedule's slot; -1: none)
  auto slot_at = [&](int n) {
    return !(ckpt && n % st->segment == 0) ? -1 : st->snap_slot ? st->snap_slot[n / st->segment] : n / st->segment;
  };
  const bool pairs = g->ndim == 2 && tu.fwd.depth == 2 && L.levels == 4;
  for (int n = n_begin; n < n_end;) {
    const int slot = slot_at(n);
    if (slot >= 0) {
      T* faces[2];
      if (pml) pml_faces<T>((T*)st->pml_psi, LE, n, faces);
      int rc = snap_store<T>(g, st, a->n_shots, L.at(n - 1), L.at(n), slot, s, pml ? faces : nullptr);
      if (rc) return rc;
    }
    T* lap = st->history ? (T*)st->history + (long long)n * LE : nullptr;
    if (pairs && n + 1 < n_end && slot_at(n + 1) < 0) {  // steps n and n+1 in one launch
      int rc = forward_pair<T>(g, kg, m, a, t, tu, L, n, true, traces, lap, lap ? lap + LE : nullptr, s);
      if (rc) return rc;
      n += 2;
      continue;
    }
    // from the second step of the call on, p^{n-1} is the output of a step two launches back
    int rc = forward_step<T>(g, kg, m, a, t, tu, L, n, traces, lap, s, (T*)st->pml_psi, n > n_begin);
    if (rc) return rc;
    ++n;
  }
  if (traces && n_end == t->n_steps && t->n_steps % t->substeps == 0) {
    int rc = launch_sample<T>(g, a, t->n_t, L.at(n_end), n_end / t->substeps, traces, s);
    if (rc) return rc;
  }
  return NW_OK;
}

// ---- adjoint driver ---------------------------------------------------------------------
int grid_blocks(long long work, int threads) {
  long long b = (work + threads - 1) / threads;
  return (int)std::max(1LL, std::min(b, 148LL * 32));
}

template <typename T>
int adjoint_impl(const nw_grid* g, const nw_medium* m, const nw_acquisition* a, const nw_time* t,
                 const nw_storage* st, const Tune& tu, const T* gtr, T* work, T* gacc, T* lambda0,
                 T* mu1, cudaStream_t s) {
  const int N = t->n_steps, M = t->substeps, S = a->n_shots;
  const long long LE = (long long)S * g->field_elems;
  const size_t lvl_bytes = (size_t)LE * sizeof(T);
  const nw::KGrid<T> kg = kgrid<T>(g);
  const bool ab = m->coef_a != nullptr;
  NW_CUDA(cudaMemsetAsync(work, 0, work_levels(g) * lvl_bytes, s));
  NW_CUDA(cudaMemsetAsync(gacc, 0, (size_t)n_acc_fields(g, tu, S) * g->field_elems * sizeof(T), s));
  auto q = [&](int n) { return work + (long long)(n % 3) * LE; };  // q^n = C mu^n, three levels
  const bool hist = st->history != nullptr;
  const bool ckpt = !hist && st->snap != nullptr;
  if (!hist && !ckpt && N > 0) return fail(NW_ERR_ARG, "adjoint needs a history or snapshots");
  const int K = ckpt ? st->segment : 0;
  if (ckpt && (K < 1 || !st->ring || !st->segbuf))
    return fail(NW_ERR_ARG, "snapshots need a ring, a segment buffer and segment >= 1");
  Ring<T> L;  // the pressure levels of the segment being recomputed
  L.base = (T*)st->ring;
  L.level_elems = LE;
  L.levels = ckpt ? ring_levels(st) : 3;
  const bool pairs = g->ndim == 2 && tu.fwd.depth == 2 && L.levels == 4;
  // forward steps [k0, k1) of a recompute or an advance; Lap p^k into seg + (k - k0) levels if seg
  auto recompute = [&](int k0, int k1, T* seg) -> int {
    for (int k = k0; k < k1;) {
      T* lp = seg ? seg + (long long)(k - k0) * LE : nullptr;
      if (pairs && k + 1 < k1) {
        const int rc = forward_pair<T>(g, kg, m, a, t, tu, L, k, true, nullptr, lp, lp ? lp + LE : nullptr, s);
        if (rc) return rc;
        k += 2;
        continue;
      }
      const int rc = forward_step<T>(g, kg, m, a, t, tu, L, k, nullptr, lp, s, (T*)st->pml_psi, k > k0);
      if (rc) return rc;
      ++k;
    }
    return NW_OK;
  };
  int seg_n0 = -1;  // first step of the segment whose Lap p levels the segment buffer holds
  const int n_stop = lambda0 ? 0 : 1;
  dim3 ig(((a->n_cells > 0 ? a->n_cells : 1) + 127) / 128, S);
  auto inject3 = [&](int n) -> int {  // 3-D: separate adjoint-source kernel
    if (a->n_cells <= 0 || n % M != 0) return NW_OK;
    return launch_pdl_b(nw::inject_kernel<T>, ig, dim3(128), 0, s, q(n), (long long)g->field_elems,
                        (const T*)m->c2dt2, (const T*)m->coef_a, n >= 1 ? 1 : 0, gtr, (int)a->n_rec, (int)t->n_t,
                        n / M, (int)a->n_cells, a->cell_index, (const int*)a->cell_ptr, (const int*)a->cell_rec,
                        (const T*)a->cell_weight);
  };
  auto step2 = [&](int n, const T* lap) -> int {  // 2-D: one fused tiled launch
    nw::Tiled2<T> as = {};
    as.cur = q(n + 1);
    as.prev = q(n + 2);
    as.next = q(n);
    as.C = (const T*)m->c2dt2;
    as.A = (const T*)m->coef_a;
    as.B = (const T*)m->coef_b;
    as.apply_a = n >= 1 ? 1 : 0;
    as.lap = lap;
    // the history was written by the forward sweep; a segment buffer level by the recompute, whose
    // last step the segment's first adjoint step (n = segment end - 1) directly follows
    as.lap_ready = hist || (K > 0 && (n + 1) % K != 0 && n + 1 != N);
    as.gacc = gacc;
    as.n_shots = S;
    as.shots_per_cta = tu.adj.spc;
    as.gtr = (a->n_cells > 0 && n % M == 0) ? gtr : nullptr;
    as.gcell_w = (const T*)a->cell_weight;
    as.n_rec = a->n_rec;
    as.n_t = t->n_t;
    as.j = n / M;
    as.tt = tile_tables(g, a, tu.adj);
    return NW_DISPATCH2(launch_adj2_v, T, tu.adj, kg, as, tu.adj.grid(g, S), s);
  };
  const bool pml = g->absorbing == NW_ABS_PML;
  if (pml && ckpt && !st->pml_psi) return fail(NW_ERR_ARG, "a checkpointed PML adjoint needs storage.pml_psi");
  auto step_pml = [&](int n, const T* lap) -> int {  // PML step (face cotangents in work levels 3..6)
    nw::PmlStep<T> ps = {};
    ps.prev = q(n + 2);
    ps.cur = q(n + 1);
    ps.next = q(n);
    pml_medium(m, ps);
    for (int ax = 0; ax < 2; ++ax) {
      ps.f_old[ax] = work + (long long)(3 + 2 * ax + (n + 1) % 2) * LE;
      ps.f_new[ax] = work + (long long)(3 + 2 * ax + n % 2) * LE;
    }
    ps.apply_a = n >= 1 ? 1 : 0;
    ps.lap = lap;
    ps.grad = gacc;
    bool box_inject = false;
    int rc = pml_tiled_box<T>(g, m, tu.adj, ps);
    if (rc) return rc;
    if (ps.kx1 == ps.kx0) {  // no interior box: the layer kernel over every cell
      rc = launch_pml<T, true>(g, kg, ps, S, s);
      if (rc) return rc;
    } else {  // the layer (per-shot accumulators) on the side stream, beside the interior box
      // the interior box: the plain adjoint step, accumulators per shot group
      nw::Tiled2<T> tb = {};  // (disjoint cells, so the reduction over all accumulators stays exact)
      tb.cur = ps.cur;
      tb.prev = ps.prev;
      tb.next = ps.next;
      tb.C = (const T*)m->c2dt2;
      tb.A = (const T*)m->coef_a;
      tb.B = (const T*)m->coef_b;
      tb.apply_a = ps.apply_a;
      tb.lap = lap;
      tb.gacc = gacc;
      // the receiver cotangents: added by the box's launch and the layer's when the adjoint tile tables
      // were built for this box's tiles (the touched cells outside it listed for the layer), else by
      // inject3 after the step
      tb.tt = tile_tables(g, a, tu.adj);
      const dim3 grid = box_tiles<T>(ps, tu.adj, S, tb);
      box_inject = box_injects(a, tu.adj, ps.kx0, ps.kz0, tb.tt.tiles_z);
      if (box_inject && n % M == 0) {  // the box's cells by the box, the layer's by the layer
        tb.gtr = gtr;
        tb.gcell_w = (const T*)a->cell_weight;
        tb.n_rec = a->n_rec;
        tb.n_t = t->n_t;
        tb.j = n / M;
        layer_inject<T>(a, gtr, t->n_t, n / M, ps);
      }
      rc = fork_join(
          s, true, [&](cudaStream_t t) { return launch_pml<T, true>(g, kg, ps, S, t); },
          [&](cudaStream_t t) { return NW_DISPATCH2(launch_adj2_v, T, tu.adj, kg, tb, grid, t); });
      if (rc) return rc;
    }
    return box_inject ? NW_OK : inject3(n);  // (inject3 itself skips the steps without cotangents)
  };
  if (N >= n_stop) {  // level N: q^N = A C R^T g_N (q^{N+1} = q^{N+2} = 0)
    int rc = pml ? step_pml(N, nullptr) : (g->ndim == 2 ? step2(N, nullptr) : inject3(N));
    if (rc) return rc;
  }
  // the binomial schedule's program (host memory), run up to the YOUTURN of each segment as the
  // adjoint reaches the segment's end
  const int32_t* prog = ckpt ? st->schedule : nullptr;
  int pc = 0;
  auto run_program = [&](int seg) -> int {
    while (pc < st->n_schedule) {
      const int op = prog[3 * pc], x = prog[3 * pc + 1], y = prog[3 * pc + 2];
      ++pc;
      T* faces[2];
      switch (op) {
        case NW_SCHED_RESTORE:
        case NW_SCHED_TAKE: {
          if (y < 0 || (long long)y * K >= N || x < 0) return fail(NW_ERR_ARG, "schedule: bad slot or segment");
          if (pml) pml_faces<T>((T*)st->pml_psi, LE, y * K, faces);
          const int rc = op == NW_SCHED_RESTORE
                             ? snap_load<T>(g, st, S, x, L.at(y * K - 1), L.at(y * K), s, pml ? faces : nullptr)
                             : snap_store<T>(g, st, S, L.at(y * K - 1), L.at(y * K), x, s, pml ? faces : nullptr);
          if (rc) return rc;
          break;
        }
        case NW_SCHED_ADVANCE: {
          if (x < 0 || y <= x || (long long)y * K >= N) return fail(NW_ERR_ARG, "schedule: bad advance");
          const int rc = recompute(x * K, y * K, nullptr);
          if (rc) return rc;
          break;
        }
        case NW_SCHED_YOUTURN:
          if (x != seg) return fail(NW_ERR_ARG, "schedule: segments must be reversed last to first, one YOUTURN each");
          return NW_OK;
        default:
          return fail(NW_ERR_ARG, "schedule: unknown operation");
      }
    }
    return fail(NW_ERR_ARG, "schedule: ended before the YOUTURN of segment " + std::to_string(seg));
  };
  for (int n = N - 1; n >= n_stop; --n) {
    const T* lap;
    if (hist) {
      lap = (const T*)st->history + (long long)n * LE;
    } else {
      const int n0 = (n / K) * K;
      if (seg_n0 != n0) {  // entering a segment from its end: recompute Lap p^{n0..n1-1}
        const int n1 = std::min(n0 + K, N);
        seg_n0 = n0;
        T* faces[2];  // with a PML the recompute runs its face fields in storage.pml_psi
        if (pml) pml_faces<T>((T*)st->pml_psi, LE, n0, faces);
        // the ring to the segment's start: the schedule's program, or the segment's own snapshot
        int rc = prog ? run_program(n0 / K)
                      : snap_load<T>(g, st, S, n0 / K, L.at(n0 - 1), L.at(n0), s, pml ? faces : nullptr);
        if (rc) return rc;
        rc = recompute(n0, n1, (T*)st->segbuf);
        if (rc) return rc;
      }
      lap = (const T*)st->segbuf + (long long)(n - n0) * LE;
    }
    if (pml) {
      int rc = step_pml(n, lap);
      if (rc) return rc;
      continue;
    }
    if (g->ndim == 2) {
      int rc = step2(n, lap);
      if (rc) return rc;
      continue;
    }
    nw::Step3<T> as = {};
    as.cur = q(n + 1);
    as.prev = q(n + 2);
    as.next = q(n);
    as.C = (const T*)m->c2dt2;
    as.A = (const T*)m->coef_a;
    as.B = (const T*)m->coef_b;
    as.apply_a = n >= 1 ? 1 : 0;
    as.lap = lap;
    as.grad = gacc;
    int rc = launch_step3<T, true>(g, kg, as, ab, S, s);
    if (rc) return rc;
    rc = inject3(n);
    if (rc) return rc;
  }
  if (lambda0) {  // lambda^0 = q^0 / C and mu^1 = q^1 / C on the padded grid, zero ghosts
    NW_CUDA(cudaMemsetAsync(lambda0, 0, lvl_bytes, s));
    const long long cells = (long long)g->n[0] * g->n[1] * (g->ndim == 3 ? g->n[2] : 1);
    dim3 ug(grid_blocks(cells, 256), S);
    nw::unscale_kernel<T><<<ug, 256, 0, s>>>(kg, g->ndim, (const T*)m->c2dt2, q(0), lambda0);
    NW_LAUNCHED();
    if (mu1) {
      NW_CUDA(cudaMemsetAsync(mu1, 0, lvl_bytes, s));
      if (N > 0) {
        nw::unscale_kernel<T><<<ug, 256, 0, s>>>(kg, g->ndim, (const T*)m->c2dt2, q(1), mu1);
        NW_LAUNCHED();
      }
    }
  }
  return NW_OK;
}

}  // namespace

// =============================================================================================
extern "C" {

int nw_abi_version(void) { return NW_ABI_VERSION; }
int nw_built_arch(void) { return 1000; }
const char* nw_last_error(void) { return g_err.c_str(); }

int nw_grid_layout(nw_grid* g) {
  if (!g) return fail(NW_ERR_ARG, "grid is NULL");
  if (g->ndim != 2 && g->ndim != 3) return fail(NW_ERR_UNSUPPORTED, "ndim must be 2 or 3");
  if (g->order != 2 && g->order != 4) return fail(NW_ERR_ARG, "order must be 2 or 4");
  const int r = g->order / 2;
  g->radius = r;
  g->guard = kGuard;
  const int last = g->ndim - 1;
  const long long ld = ((long long)g->n[last] + r + 31) / 32 * 32;
  if (g->ndim == 2) {
    g->stride[0] = ld;
    g->stride[1] = 1;
    g->stride[2] = 0;
    g->origin = kGuard + (long long)r * ld;
    g->field_elems = kGuard + ((long long)g->n[0] + 2 * r) * ld;
  } else {
    const long long rows = (long long)g->n[1] + r;
    g->stride[0] = rows * ld;
    g->stride[1] = ld;
    g->stride[2] = 1;
    g->origin = kGuard + (long long)r * rows * ld;
    g->field_elems = kGuard + ((long long)g->n[0] + 2 * r) * rows * ld;
  }
  return NW_OK;
}

size_t nw_snapshot_bytes(const nw_grid* g, int32_t n_shots, int32_t n_snap, int32_t snap_kind) {
  if (!g || n_shots < 1 || n_snap < 0) return 0;
  return snap_layout(g, n_shots).per_snap(snap_kind) * (size_t)n_snap;
}

int nw_prepare_medium(const nw_grid* g, const int32_t* n_abs, const void* c, double dt2, void* c2dt2,
                      void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!c || !c2dt2 || !n_abs) return fail(NW_ERR_ARG, "NULL pointer");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t esz = g->dtype == NW_F64 ? 8 : 4;
  NW_CUDA(cudaMemsetAsync(c2dt2, 0, g->field_elems * esz, s));
  const nw::PadMap pm = padmap(g, n_abs);
  const long long cells = (long long)g->n[0] * g->n[1] * (g->ndim == 3 ? g->n[2] : 1);
  const int blocks = grid_blocks(cells, 256);
  if (g->dtype == NW_F32)
    nw::medium_kernel<float><<<blocks, 256, 0, s>>>(kgrid<float>(g), pm, (const float*)c, (float)dt2,
                                                    g->ndim, (float*)c2dt2);
  else
    nw::medium_kernel<double><<<blocks, 256, 0, s>>>(kgrid<double>(g), pm, (const double*)c, dt2,
                                                     g->ndim, (double*)c2dt2);
  NW_LAUNCHED();
  return NW_OK;
}

int nw_initial_state(const nw_grid* g, const int32_t* n_abs, const nw_medium* m, int32_t n_shots,
                     const void* p0, void* pm1_level, void* p0_level, void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!m || !p0 || !pm1_level || !p0_level || !n_abs || n_shots < 1)
    return fail(NW_ERR_ARG, "invalid initial-state arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t esz = g->dtype == NW_F64 ? 8 : 4;
  const size_t lvl = (size_t)n_shots * g->field_elems * esz;
  NW_CUDA(cudaMemsetAsync(p0_level, 0, lvl, s));
  NW_CUDA(cudaMemsetAsync(pm1_level, 0, lvl, s));
  const nw::PadMap pm = padmap(g, n_abs);
  const long long pcells = (long long)pm.m0 * pm.m1 * pm.m2;
  const long long cells = (long long)g->n[0] * g->n[1] * (g->ndim == 3 ? g->n[2] : 1);
  dim3 gp(grid_blocks(pcells, 256), n_shots), gc(grid_blocks(cells, 256), n_shots);
  if (g->dtype == NW_F32) {
    auto kg = kgrid<float>(g);
    nw::pad_zero_kernel<float><<<gp, 256, 0, s>>>(kg, pm, g->ndim, (const float*)p0, (float*)p0_level);
    if (g->radius == 1)
      nw::initial_prev_kernel<float, 1><<<gc, 256, 0, s>>>(kg, g->ndim, (const float*)m->c2dt2,
                                                          (const float*)p0_level, (float*)pm1_level);
    else
      nw::initial_prev_kernel<float, 2><<<gc, 256, 0, s>>>(kg, g->ndim, (const float*)m->c2dt2,
                                                          (const float*)p0_level, (float*)pm1_level);
  } else {
    auto kg = kgrid<double>(g);
    nw::pad_zero_kernel<double><<<gp, 256, 0, s>>>(kg, pm, g->ndim, (const double*)p0, (double*)p0_level);
    if (g->radius == 1)
      nw::initial_prev_kernel<double, 1><<<gc, 256, 0, s>>>(kg, g->ndim, (const double*)m->c2dt2,
                                                           (const double*)p0_level, (double*)pm1_level);
    else
      nw::initial_prev_kernel<double, 2><<<gc, 256, 0, s>>>(kg, g->ndim, (const double*)m->c2dt2,
                                                           (const double*)p0_level, (double*)pm1_level);
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);  // pad_zero_kernel
  NW_LAUNCHED();
  return NW_OK;
}

// The step kernels and the snapshot codecs move fields in 16-byte vectors.
static bool misaligned16(const void* p) { return ((uintptr_t)p & 15u) != 0; }

static int check_run(const nw_grid* g, const nw_medium* m, const nw_acquisition* a, const nw_time* t,
                     const nw_storage* st, const Tune& tu) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!m || !a || !t || !st) return fail(NW_ERR_ARG, "NULL descriptor");
  if (!m->c2dt2) return fail(NW_ERR_ARG, "medium.c2dt2 is NULL");
  if (misaligned16(m->c2dt2) || misaligned16(m->coef_a) || misaligned16(m->coef_b) ||
      misaligned16(st->history) || misaligned16(st->ring) || misaligned16(st->snap) ||
      misaligned16(st->segbuf) || misaligned16(st->pml_psi))
    return fail(NW_ERR_ARG, "device buffers must start on 16-byte boundaries");
  if ((g->absorbing != NW_ABS_NONE) != (m->coef_a != nullptr) || (m->coef_a == nullptr) != (m->coef_b == nullptr))
    return fail(NW_ERR_ARG, "absorbing coefficients must be given exactly when absorbing != none");
  if (a->n_shots < 1) return fail(NW_ERR_ARG, "n_shots must be >= 1");
  if (a->n_shots > 65535) return fail(NW_ERR_ARG, "n_shots must be <= 65535");
  if (a->has_source && (!a->src_corner || !a->src_weight || !a->wavelet))
    return fail(NW_ERR_ARG, "source arrays are NULL");
  if (a->n_rec > 0 && (!a->rec_index || !a->rec_weight)) return fail(NW_ERR_ARG, "receiver arrays are NULL");
  if (t->substeps < 1 || t->n_t < 1 || t->n_steps != (t->n_t - 1) * t->substeps)
    return fail(NW_ERR_ARG, "inconsistent time axis");
  if (a->adj_tables_box && (g->ndim != 2 || g->absorbing != NW_ABS_PML))
    return fail(NW_ERR_ARG, "adjoint tables of a PML's interior box on a grid without a PML");
  if (g->ndim == 2) {
    // (tables of a PML's interior box count its tiles only; box_injects checks them before use)
    if (a->tile_rows != tu.fwd.tx() || a->tile_cols != tu.fwd.tz() || a->tiles_z != tu.fwd.tiles_z(g) ||
        a->adj_tile_rows != tu.adj.tx() || a->adj_tile_cols != tu.adj.tz() ||
        (!a->adj_tables_box && a->adj_tiles_z != tu.adj.tiles_z(g)))
      return fail(NW_ERR_ARG, "per-tile tables were built for another tile shape (see nw_tile_shape)");
    if (!a->tile_rec_ptr || !a->tile_cell_ptr || !a->rec_corner ||
        (a->n_cells > 0 && (!a->tile_cell_local || !a->tile_cell_gid)) || (a->n_rec > 0 && !a->tile_rec_list))
      return fail(NW_ERR_ARG, "2-D grids need the per-tile receiver tables");
  }
  return NW_OK;
}

int nw_tile_shape(const nw_grid* g, nw_tuning* t, int32_t* shape) {
  int rc = check_grid(g);
  if (rc) return rc;
  Tune tu;
  rc = resolve_tune(g, t, &tu);
  if (rc) return rc;
  if (t) {
    t->vz = tu.fwd.vz;
    t->rx = tu.fwd.rx;
    t->shots_per_cta = tu.fwd.spc;
    t->adj_vz = tu.adj.vz;
    t->adj_rx = tu.adj.rx;
    t->adj_shots_per_cta = tu.adj.spc;
  }
  if (shape) {
    shape[0] = tu.fwd.tx();
    shape[1] = tu.fwd.tz();
    shape[2] = tu.adj.tx();
    shape[3] = tu.adj.tz();
  }
  return NW_OK;
}

int nw_adjoint_groups(const nw_grid* g, const nw_tuning* t, int32_t n_shots) {
  Tune tu;
  if (check_grid(g) || resolve_tune(g, t, &tu) || n_shots < 1) return -1;
  return n_acc_fields(g, tu, n_shots);
}

int nw_forward(const nw_grid* g, const nw_medium* m, const nw_acquisition* a, const nw_time* t,
               const nw_storage* st, const nw_tuning* tune, int32_t n_begin, int32_t n_end, void* traces,
               void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  Tune tu;
  rc = resolve_tune(g, tune, &tu);
  if (rc) return rc;
  rc = check_run(g, m, a, t, st, tu);
  if (rc) return rc;
  if (n_begin < 0 || n_end < n_begin || n_end > t->n_steps) return fail(NW_ERR_ARG, "step range out of bounds");
  if (g->dtype == NW_F32)
    return forward_impl<float>(g, m, a, t, st, tu, n_begin, n_end, (float*)traces, (cudaStream_t)stream);
  return forward_impl<double>(g, m, a, t, st, tu, n_begin, n_end, (double*)traces, (cudaStream_t)stream);
}

int nw_adjoint(const nw_grid* g, const nw_medium* m, const nw_acquisition* a, const nw_time* t,
               const nw_storage* st, const nw_tuning* tune, const void* grad_traces, void* work,
               void* grad_acc, void* lambda0, void* mu1, void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  Tune tu;
  rc = resolve_tune(g, tune, &tu);
  if (rc) return rc;
  rc = check_run(g, m, a, t, st, tu);
  if (rc) return rc;
  if (!grad_traces || !work || !grad_acc) return fail(NW_ERR_ARG, "NULL adjoint buffer");
  if (misaligned16(work) || misaligned16(grad_acc) || misaligned16(lambda0) || misaligned16(mu1))
    return fail(NW_ERR_ARG, "device buffers must start on 16-byte boundaries");
  if (a->n_cells > 0 && (!a->cell_index || !a->cell_ptr || !a->cell_rec || !a->cell_weight))
    return fail(NW_ERR_ARG, "receiver adjoint table is NULL");
  if (!st->history && st->snap && !st->segbuf) return fail(NW_ERR_ARG, "checkpointing needs segbuf");
  if (g->dtype == NW_F32)
    return adjoint_impl<float>(g, m, a, t, st, tu, (const float*)grad_traces, (float*)work, (float*)grad_acc,
                               (float*)lambda0, (float*)mu1, (cudaStream_t)stream);
  return adjoint_impl<double>(g, m, a, t, st, tu, (const double*)grad_traces, (double*)work, (double*)grad_acc,
                              (double*)lambda0, (double*)mu1, (cudaStream_t)stream);
}

int nw_reduce_grad_c(const nw_grid* g, const int32_t* n_abs, const void* c, double dt2,
                     int32_t n_acc, const void* grad_acc, int32_t accumulate, double* grad_c,
                     void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!n_abs || !c || !grad_acc || !grad_c || n_acc < 1) return fail(NW_ERR_ARG, "invalid reduce arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const nw::PadMap pm = padmap(g, n_abs);
  const long long pcells = (long long)pm.m0 * pm.m1 * pm.m2;
  const int blocks = grid_blocks(pcells, 128);
  if (g->dtype == NW_F32)
    nw::reduce_grad_kernel<float><<<blocks, 128, 0, s>>>(kgrid<float>(g), pm, g->ndim, (const float*)c, dt2,
                                                         n_acc, (const float*)grad_acc, accumulate, grad_c);
  else
    nw::reduce_grad_kernel<double><<<blocks, 128, 0, s>>>(kgrid<double>(g), pm, g->ndim, (const double*)c,
                                                          dt2, n_acc, (const double*)grad_acc, accumulate, grad_c);
  NW_LAUNCHED();
  return NW_OK;
}

int nw_initial_state_adjoint(const nw_grid* g, const int32_t* n_abs, const nw_medium* m,
                             const nw_time* t, int32_t n_shots, const void* lambda0,
                             const void* mu1, const void* p0_level, void* grad_p0,
                             void* grad_acc, int32_t shots_per_acc, void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!m || !t || !n_abs || !lambda0 || !mu1 || !p0_level || !grad_p0 || n_shots < 1 || shots_per_acc < 1)
    return fail(NW_ERR_ARG, "invalid initial-state adjoint arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const nw::PadMap pm = padmap(g, n_abs);
  const long long cells = (long long)g->n[0] * g->n[1] * (g->ndim == 3 ? g->n[2] : 1);
  const int groups = (n_shots + shots_per_acc - 1) / shots_per_acc;
  dim3 gc(grid_blocks(cells, 256), groups);
  const int b_one = t->first_b_one;
#define NW_IA(T, R)                                                                                       \
  nw::initial_adjoint_kernel<T, R><<<gc, 256, 0, s>>>(kgrid<T>(g), pm, g->ndim, (const T*)m->c2dt2,       \
                                                      (const T*)m->coef_b, b_one, n_shots, shots_per_acc, \
                                                      (const T*)lambda0, (const T*)mu1, (const T*)p0_level, \
                                                      (T*)grad_p0, (T*)grad_acc)
  if (g->dtype == NW_F32) { if (g->radius == 1) NW_IA(float, 1); else NW_IA(float, 2); }
  else { if (g->radius == 1) NW_IA(double, 1); else NW_IA(double, 2); }
#undef NW_IA
  NW_LAUNCHED();
  return NW_OK;
}

int nw_sample(const nw_grid* g, const nw_acquisition* a, int32_t n_t, const void* level, int32_t j,
              void* traces, void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!a || !level || !traces || j < 0 || j >= n_t) return fail(NW_ERR_ARG, "invalid sample arguments");
  if (g->dtype == NW_F32)
    return launch_sample<float>(g, a, n_t, (const float*)level, j, (float*)traces, (cudaStream_t)stream);
  return launch_sample<double>(g, a, n_t, (const double*)level, j, (double*)traces, (cudaStream_t)stream);
}

int nw_zero_ghosts(const nw_grid* g, void* fields, int64_t n_fields, void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!fields || n_fields < 0) return fail(NW_ERR_ARG, "invalid zero_ghosts arguments");
  if (n_fields == 0) return NW_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int last = g->ndim - 1;
  const int ld = (int)g->stride[last - 1];
  const long long n_rows = (g->field_elems - g->guard) / ld;
  const int rows_per_plane = g->ndim == 3 ? (int)(g->stride[0] / g->stride[1]) : 1;
  const int blocks = grid_blocks(n_rows * n_fields * 32, 256);
  if (g->dtype == NW_F32)
    nw::zero_ghosts_kernel<float><<<blocks, 256, 0, s>>>((float*)fields, g->field_elems, g->guard, n_rows, ld,
                                                         g->n[last], g->ndim, g->radius, g->n[0], g->n[1],
                                                         rows_per_plane, n_fields);
  else
    nw::zero_ghosts_kernel<double><<<blocks, 256, 0, s>>>((double*)fields, g->field_elems, g->guard, n_rows, ld,
                                                          g->n[last], g->ndim, g->radius, g->n[0], g->n[1],
                                                          rows_per_plane, n_fields);
  NW_LAUNCHED();
  return NW_OK;
}

uint64_t nw_launch_count(void) { return g_launches.load(); }

// Synchronises `stream`, returns and clears the sticky device status word (NW_OK if clean).
int nw_status(void* stream) {
  NW_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  int v = 0;
  NW_CUDA(cudaMemcpyFromSymbol(&v, nw::g_status, sizeof(int)));
  if (v) {
    const int zero = 0;
    NW_CUDA(cudaMemcpyToSymbol(nw::g_status, &zero, sizeof(int)));
    return fail(v, "a snapshot block held a non-finite value or scale");
  }
  return NW_OK;
}

}  // extern "C"

// =============================================================================================
// Allocation-free adjoint gradient: nw_adjoint + nw_reduce_grad_c with their scratch (the three
// adjoint levels and the gradient accumulators) carved out of a fixed array in device memory
// instead of caller buffers. The array is module-scope device storage, so every GPU that loads
// this library holds NW_NOALLOC_SCRATCH_BYTES of it until the process exits.
// =============================================================================================
namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[NW_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 128;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device. The host symbol is only a
// stand-in, so the address is looked up once per device (with that device current) and cached.
int noalloc_scratch(void** out) {
  int dev = 0;
  NW_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(NW_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    NW_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return NW_OK;
}

template <typename T>
int noalloc_gradient(const nw_grid* g, const int32_t* n_abs, const nw_medium* m, const nw_acquisition* a,
                     const nw_time* t, const nw_storage* st, const Tune& tu, const void* c, double dt2,
                     const T* gtr, double* grad_c, cudaStream_t s) {
  const size_t work_bytes = (size_t)work_levels(g) * a->n_shots * g->field_elems * sizeof(T);
  const size_t acc_off = (work_bytes + 255) / 256 * 256;
  const int n_acc = n_acc_fields(g, tu, a->n_shots);
  const size_t need = acc_off + (size_t)n_acc * g->field_elems * sizeof(T);
  if (need > NW_NOALLOC_SCRATCH_BYTES)
    return fail(NW_ERR_ARG, "nw_adjoint_grad_c_noalloc needs " + std::to_string(need) +
                                " bytes of scratch, above its fixed " + std::to_string(NW_NOALLOC_SCRATCH_BYTES) +
                                "-byte array; use nw_adjoint with caller-allocated buffers or fewer shots per call");
  void* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  T* work = reinterpret_cast<T*>(base);
  T* acc = reinterpret_cast<T*>(reinterpret_cast<char*>(base) + acc_off);
  // adjoint_impl clears the work levels and the accumulators on `s` before using them, so the
  // previous call's contents never leak into this one.
  rc = adjoint_impl<T>(g, m, a, t, st, tu, gtr, work, acc, nullptr, nullptr, s);
  if (rc) return rc;
  const nw::PadMap pm = padmap(g, n_abs);
  const long long pcells = (long long)pm.m0 * pm.m1 * pm.m2;
  nw::reduce_grad_kernel<T><<<grid_blocks(pcells, 128), 128, 0, s>>>(kgrid<T>(g), pm, g->ndim, (const T*)c, dt2,
                                                                     n_acc, acc, 0, grad_c);
  NW_LAUNCHED();
  return NW_OK;
}

}  // namespace

extern "C" int nw_adjoint_grad_c_noalloc(const nw_grid* g, const int32_t* n_abs, const nw_medium* m,
                                         const nw_acquisition* a, const nw_time* t, const nw_storage* st,
                                         const nw_tuning* tune, const void* c, double dt2,
                                         const void* grad_traces, double* grad_c, void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  Tune tu;
  rc = resolve_tune(g, tune, &tu);
  if (rc) return rc;
  rc = check_run(g, m, a, t, st, tu);
  if (rc) return rc;
  if (!n_abs || !c || !grad_traces || !grad_c) return fail(NW_ERR_ARG, "NULL argument");
  if (a->n_cells > 0 && (!a->cell_index || !a->cell_ptr || !a->cell_rec || !a->cell_weight))
    return fail(NW_ERR_ARG, "receiver adjoint table is NULL");
  if (!st->history && st->snap && !st->segbuf) return fail(NW_ERR_ARG, "checkpointing needs segbuf");
  if (g->dtype == NW_F32)
    return noalloc_gradient<float>(g, n_abs, m, a, t, st, tu, c, dt2, (const float*)grad_traces, grad_c,
                                   (cudaStream_t)stream);
  return noalloc_gradient<double>(g, n_abs, m, a, t, st, tu, c, dt2, (const double*)grad_traces, grad_c,
                                  (cudaStream_t)stream);
}

// =============================================================================================
// Batched problems (nw_batch_*): the device table is [BatchProb x n][fwd CTA offsets x (n+1)]
// [adj CTA offsets x (n+1)]; the CTA offsets are prefix sums over the problems in table order,
// which is non-increasing step count, so the problems taking part in step n are a prefix.
// =============================================================================================
namespace {

struct BatchLayout {
  size_t fcta, acta, bytes;
};
BatchLayout batch_layout(int n) {
  BatchLayout L;
  const size_t probs = ((sizeof(nw::BatchProb<double>) * (size_t)n + 255) / 256) * 256;
  L.fcta = probs;
  L.acta = L.fcta + ((sizeof(int) * (size_t)(n + 1) + 255) / 256) * 256;
  L.bytes = L.acta + ((sizeof(int) * (size_t)(n + 1) + 255) / 256) * 256;
  return L;
}

int check_batch(const nw_batch_problem* P, int n, const Tune& tu) {
  if (!P || n < 1) return fail(NW_ERR_ARG, "empty batch");
  for (int p = 0; p < n; ++p) {
    const nw_batch_problem& q = P[p];
    int rc = check_run(&q.grid, &q.medium, &q.acq, &q.time, &q.storage, tu);
    if (rc) return fail(rc, "batch problem " + std::to_string(p) + ": " + g_err);
    if (q.grid.ndim != 2) return fail(NW_ERR_UNSUPPORTED, "batched problems are 2-D");
    if (q.grid.absorbing == NW_ABS_PML && !q.storage.pml_psi)
      return fail(NW_ERR_ARG, "batch problem " + std::to_string(p) + " has a PML but no storage.pml_psi");
    if (q.grid.dtype != P[0].grid.dtype || q.grid.order != P[0].grid.order)
      return fail(NW_ERR_ARG, "batched problems share one dtype and stencil order");
    if (!q.acq.has_source) return fail(NW_ERR_UNSUPPORTED, "batched problems are FWI problems (with sources)");
    if (!q.storage.ring || !q.storage.snap || !q.storage.segbuf || q.storage.history)
      return fail(NW_ERR_ARG, "batched problems use checkpointed storage (ring, snapshots, segment buffer)");
    if (q.storage.segment != P[0].storage.segment || q.storage.snap_kind != P[0].storage.snap_kind ||
        q.storage.segment < 1)
      return fail(NW_ERR_ARG, "batched problems share one segment length >= 1 and snapshot kind");
    if (p > 0 && q.time.n_steps > P[p - 1].time.n_steps)
      return fail(NW_ERR_ARG, "batched problems must be ordered by non-increasing n_steps");
    if (!q.work || !q.grad_acc || !q.traces || (q.acq.n_cells > 0 && !q.grad_traces))
      return fail(NW_ERR_ARG, "batch problem " + std::to_string(p) + " lacks a work, accumulator or trace buffer");
  }
  return NW_OK;
}

// The tiles a batched launch steps for problem q: the whole grid, or with a PML the interior box
// (the layer goes through the PML kernel in launches of its own). The box depends on T only through
// its 16-byte column alignment, which the batch's dtype fixes.
template <typename T>
dim3 batch_grid(const nw_batch_problem& q, const TileCfg& c) {
  if (q.grid.absorbing != NW_ABS_PML) return c.grid(&q.grid, q.acq.n_shots);
  nw::PmlStep<T> st = {};
  if (pml_tiled_box<T>(&q.grid, &q.medium, c, st) || st.kx1 == st.kx0) return dim3(0, 0, 0);
  nw::Tiled2<T> tb = {};
  return box_tiles<T>(st, c, q.acq.n_shots, tb);
}

template <typename T>
int batch_prepare_impl(const nw_batch_problem* P, int n, const Tune& tu, void* table, cudaStream_t s) {
  const BatchLayout L = batch_layout(n);
  std::vector<char> host(L.bytes, 0);
  auto* probs = reinterpret_cast<nw::BatchProb<T>*>(host.data());
  int* fcta = reinterpret_cast<int*>(host.data() + L.fcta);
  int* acta = reinterpret_cast<int*>(host.data() + L.acta);
  long long fsum = 0, asum = 0;
  for (int p = 0; p < n; ++p) {
    const nw_batch_problem& q = P[p];
    const nw_grid* g = &q.grid;
    const nw_acquisition* a = &q.acq;
    nw::BatchProb<T>& B = probs[p];
    B.g = kgrid<T>(g);
    nw::Tiled2<T> f = {};
    f.C = (const T*)q.medium.c2dt2;
    f.A = (const T*)q.medium.coef_a;
    f.B = (const T*)q.medium.coef_b;
    f.n_shots = a->n_shots;
    f.src_corner = a->src_corner;
    f.src_w = (const T*)a->src_weight;
    f.wavelet = (const T*)a->wavelet;
    f.rec_w = (const T*)a->rec_weight;
    f.gcell_w = (const T*)a->cell_weight;
    f.n_rec = a->n_rec;
    f.n_t = q.time.n_t;
    f.x_end = g->n[0];
    f.z_end = g->n[1];
    nw::Tiled2<T> b = f;
    f.shots_per_cta = tu.fwd.spc;
    f.tt = tile_tables(g, a, tu.fwd);
    b.shots_per_cta = tu.adj.spc;
    b.tt = tile_tables(g, a, tu.adj);
    b.gtr = a->n_cells > 0 ? (const T*)q.grad_traces : nullptr;
    b.gacc = (T*)q.grad_acc;
    B.fwd = f;
    B.adj = b;
    B.ring = (T*)q.storage.ring;
    B.work = (T*)q.work;
    B.segbuf = (T*)q.storage.segbuf;
    B.traces = (T*)q.traces;
    B.level = (long long)a->n_shots * g->field_elems;
    B.n_steps = q.time.n_steps;
    B.substeps = q.time.substeps;
    B.first_b_one = q.time.first_b_one;
    if (g->absorbing == NW_ABS_PML) {  // the interior box only: no receivers or cotangents in it
      nw::PmlStep<T> sf = {}, sa = {};
      int rc = pml_tiled_box<T>(g, &q.medium, tu.fwd, sf);
      if (rc) return rc;
      rc = pml_tiled_box<T>(g, &q.medium, tu.adj, sa);
      if (rc) return rc;
      nw::Tiled2<T> tf = {}, ta = {};
      box_tiles<T>(sf, tu.fwd, a->n_shots, tf);
      box_tiles<T>(sa, tu.adj, a->n_shots, ta);
      for (auto* d : {&B.fwd, &B.adj}) d->n_rec = 0;
      B.adj.gtr = nullptr;
      B.fwd.tx_off = tf.tx_off; B.fwd.tz_off = tf.tz_off; B.fwd.x_end = tf.x_end; B.fwd.z_end = tf.z_end;
      B.fwd.tt.tiles_z = tf.tt.tiles_z;
      B.adj.tx_off = ta.tx_off; B.adj.tz_off = ta.tz_off; B.adj.x_end = ta.x_end; B.adj.z_end = ta.z_end;
      B.adj.tt.tiles_z = ta.tt.tiles_z;
      if (box_injects(a, tu.adj, ta.tx_off, ta.tz_off, ta.tt.tiles_z)) {  // the box adds the cotangents
        B.adj.gtr = (const T*)q.grad_traces;
        B.adj.n_rec = a->n_rec;
      }
    }
    const dim3 fg = batch_grid<T>(q, tu.fwd), ag = batch_grid<T>(q, tu.adj);
    B.ftx = (int)fg.y;
    B.atx = (int)ag.y;
    fcta[p] = (int)fsum;
    acta[p] = (int)asum;
    fsum += (long long)fg.x * fg.y * fg.z;
    asum += (long long)ag.x * ag.y * ag.z;
    if (fsum > INT32_MAX || asum > INT32_MAX) return fail(NW_ERR_ARG, "batch too large for one launch");
  }
  fcta[n] = (int)fsum;
  acta[n] = (int)asum;
  NW_CUDA(cudaMemcpyAsync(table, host.data(), L.bytes, cudaMemcpyHostToDevice, s));
  NW_CUDA(cudaStreamSynchronize(s));  // the host staging copy dies with this call
  return NW_OK;
}

// Problems taking part in step n: forward (n_steps > n) or adjoint (n_steps >= n).
int batch_active(const nw_batch_problem* P, int n, int step, bool adjoint) {
  int k = 0;
  while (k < n && (adjoint ? P[k].time.n_steps >= step : P[k].time.n_steps > step)) ++k;
  return k;
}

template <typename T, int R, int VZ, int RX>
int launch_fwd_batch(const void* table, int n, int n_active, int n_ctas, int step, int store_lap, int segment,
                     cudaStream_t s) {
  const BatchLayout L = batch_layout(n);
  const char* base = (const char*)table;
  constexpr size_t smem = step2_smem<T, R, VZ, RX, false>();
  if (smem > kMaxSmem) return fail(NW_ERR_ARG, "tile too large for shared memory (lower tuning rx or vz)");
  static bool done = false;
  int rc = allow_smem(nw::fwd2d_batch<T, R, VZ, RX>, smem, &done);
  if (rc) return rc;
  if (n_ctas == 0) return NW_OK;  // only PML problems whose interior is smaller than a tile
  return launch_pdl(nw::fwd2d_batch<T, R, VZ, RX>, dim3(n_ctas, 1, 1), smem, s, (const nw::BatchProb<T>*)base,
                    (const int*)(base + L.fcta), n_active, step, store_lap, segment);
}
template <typename T, int R, int VZ, int RX>
int launch_adj_batch(const void* table, int n, int n_active, int n_ctas, int step, int store_lap, int segment,
                     cudaStream_t s) {
  const BatchLayout L = batch_layout(n);
  const char* base = (const char*)table;
  (void)store_lap;
  constexpr size_t smem = step2_smem<T, R, VZ, RX, true>();
  if (smem > kMaxSmem) return fail(NW_ERR_ARG, "tile too large for shared memory (lower tuning adj_rx or adj_vz)");
  static bool done = false;
  int rc = allow_smem(nw::adj2d_batch<T, R, VZ, RX>, smem, &done);
  if (rc) return rc;
  if (n_ctas == 0) return NW_OK;  // only PML problems whose interior is smaller than a tile
  return launch_pdl(nw::adj2d_batch<T, R, VZ, RX>, dim3(n_ctas, 1, 1), smem, s, (const nw::BatchProb<T>*)base,
                    (const int*)(base + L.acta), n_active, step, segment);
}

// (radius, vz, rx) -> batched kernel instantiation; batches take rx 2 or 4.
#define NW_DISPATCH_BATCH(FN, T, TU, R_, ...)                                                      \
  [&]() -> int {                                                                                  \
    if (TU.rx != 2 && TU.rx != 4) return fail(NW_ERR_UNSUPPORTED, "batched steps take rx 2 or 4"); \
    if constexpr (sizeof(T) == 4) {                                                               \
      if (TU.vz == 4) {                                                                           \
        if (R_ == 2) return TU.rx == 2 ? FN<T, 2, 4, 2>(__VA_ARGS__) : FN<T, 2, 4, 4>(__VA_ARGS__); \
        return TU.rx == 2 ? FN<T, 1, 4, 2>(__VA_ARGS__) : FN<T, 1, 4, 4>(__VA_ARGS__);            \
      }                                                                                           \
    }                                                                                             \
    if (R_ == 2) return TU.rx == 2 ? FN<T, 2, 2, 2>(__VA_ARGS__) : FN<T, 2, 2, 4>(__VA_ARGS__);   \
    return TU.rx == 2 ? FN<T, 1, 2, 2>(__VA_ARGS__) : FN<T, 1, 2, 4>(__VA_ARGS__);                \
  }()

// Host copy of the CTA offsets: cta[p] = CTAs of the problems before p.
template <typename T>
std::vector<int> batch_ctas(const nw_batch_problem* P, int n, const TileCfg& c) {
  std::vector<int> cta(n + 1, 0);
  for (int p = 0; p < n; ++p) {
    const dim3 gr = batch_grid<T>(P[p], c);
    cta[p + 1] = cta[p] + (int)(gr.x * gr.y * gr.z);
  }
  return cta;
}

template <typename T>
T* ring_level(const nw_batch_problem& q, int level) {  // pressure level `level` (>= -1) in the ring
  return (T*)q.storage.ring + (long long)((level + 1) % 3) * q.acq.n_shots * q.grid.field_elems;
}

// The PML layer of batch problem q at forward step k (its interior box is in the batched launch);
// store_lap: a recompute step that stores the step's Lap p into the segment buffer.
template <typename T>
int batch_pml_forward(const nw_batch_problem& q, const Tune& tu, int k, bool store_lap, cudaStream_t s) {
  const nw_grid* g = &q.grid;
  const long long LE = (long long)q.acq.n_shots * g->field_elems;
  nw::PmlStep<T> st = {};
  st.prev = ring_level<T>(q, k - 1);
  st.cur = ring_level<T>(q, k);
  st.next = ring_level<T>(q, k + 1);
  pml_medium(&q.medium, st);
  T* psi = (T*)q.storage.pml_psi;
  for (int ax = 0; ax < 2; ++ax) {
    st.f_old[ax] = psi + (long long)(2 * ax + k % 2) * LE;
    st.f_new[ax] = psi + (long long)(2 * ax + (k + 1) % 2) * LE;
  }
  st.src_corner = q.acq.src_corner;
  st.src_w = (const T*)q.acq.src_weight;
  st.wavelet = (const T*)q.acq.wavelet;
  st.n = k;
  st.lap_out = store_lap ? (T*)q.storage.segbuf + (long long)(k % q.storage.segment) * LE : nullptr;
  int rc = pml_tiled_box<T>(g, &q.medium, tu.fwd, st);
  if (rc) return rc;
  return launch_pml<T, false>(g, kgrid<T>(g), st, q.acq.n_shots, s);
}

// The PML layer of batch problem q at adjoint step n.
template <typename T>
int batch_pml_adjoint(const nw_batch_problem& q, const Tune& tu, int n, cudaStream_t s) {
  const nw_grid* g = &q.grid;
  const long long LE = (long long)q.acq.n_shots * g->field_elems;
  T* work = (T*)q.work;
  auto lv = [&](int m) { return work + (long long)(m % 3) * LE; };
  nw::PmlStep<T> ps = {};
  ps.prev = lv(n + 2);
  ps.cur = lv(n + 1);
  ps.next = lv(n);
  pml_medium(&q.medium, ps);
  for (int ax = 0; ax < 2; ++ax) {
    ps.f_old[ax] = work + (long long)(3 + 2 * ax + (n + 1) % 2) * LE;
    ps.f_new[ax] = work + (long long)(3 + 2 * ax + n % 2) * LE;
  }
  ps.apply_a = n >= 1 ? 1 : 0;
  ps.lap = n < q.time.n_steps ? (const T*)q.storage.segbuf + (long long)(n % q.storage.segment) * LE : nullptr;
  ps.grad = (T*)q.grad_acc;
  int rc = pml_tiled_box<T>(g, &q.medium, tu.adj, ps);
  if (rc) return rc;
  if (ps.kx1 > ps.kx0 && q.acq.n_cells > 0 && n % q.time.substeps == 0) {
    nw::Tiled2<T> ta = {};
    box_tiles<T>(ps, tu.adj, q.acq.n_shots, ta);
    if (box_injects(&q.acq, tu.adj, ta.tx_off, ta.tz_off, ta.tt.tiles_z))  // the layer's touched cells
      layer_inject<T>(&q.acq, (const T*)q.grad_traces, q.time.n_t, n / q.time.substeps, ps);
  }
  return launch_pml<T, true>(g, kgrid<T>(g), ps, q.acq.n_shots, s);
}

// The receiver cotangents of batch problem q at adjoint step n at every cell (a PML problem's
// batched launch skips them), after its interior box and layer cells.
template <typename T>
int batch_pml_inject(const nw_batch_problem& q, const Tune& tu, int n, cudaStream_t s) {
  const nw_grid* g = &q.grid;
  const long long LE = (long long)q.acq.n_shots * g->field_elems;
  T* work = (T*)q.work;
  auto lv = [&](int m) { return work + (long long)(m % 3) * LE; };
  const nw_acquisition* a = &q.acq;
  const int M = q.time.substeps;
  if (a->n_cells <= 0 || n % M != 0) return NW_OK;
  {  // the batched launch of the problem's interior box added them
    nw::PmlStep<T> sa = {};
    nw::Tiled2<T> ta = {};
    if (pml_tiled_box<T>(g, &q.medium, tu.adj, sa) == NW_OK && sa.kx1 > sa.kx0) {
      box_tiles<T>(sa, tu.adj, a->n_shots, ta);
      if (box_injects(a, tu.adj, ta.tx_off, ta.tz_off, ta.tt.tiles_z)) return NW_OK;
    }
  }
  const dim3 ig((a->n_cells + 127) / 128, a->n_shots);
  return launch_pdl_b(nw::inject_kernel<T>, ig, dim3(128), 0, s, lv(n), (long long)g->field_elems,
                      (const T*)q.medium.c2dt2, (const T*)q.medium.coef_a, n >= 1 ? 1 : 0, (const T*)q.grad_traces,
                      (int)a->n_rec, (int)q.time.n_t, n / M, (int)a->n_cells, a->cell_index, (const int*)a->cell_ptr,
                      (const int*)a->cell_rec, (const T*)a->cell_weight);
}

// Face fields of batch problem q that step k reads (PML only).
template <typename T>
void batch_pml_faces(const nw_batch_problem& q, int k, T* out[2]) {
  pml_faces<T>((T*)q.storage.pml_psi, (long long)q.acq.n_shots * q.grid.field_elems, k, out);
}

template <typename T>
int batch_forward_impl(const nw_batch_problem* P, int n, const Tune& tu, const void* table, cudaStream_t s) {
  const int K = P[0].storage.segment, Nmax = P[0].time.n_steps, R = P[0].grid.radius;
  const std::vector<int> cta = batch_ctas<T>(P, n, tu.fwd);
  for (int p = 0; p < n; ++p) {  // p^-1 = p^0 = 0 (FWI), and the PML's face fields
    const size_t lvl = (size_t)P[p].acq.n_shots * P[p].grid.field_elems * sizeof(T);
    NW_CUDA(cudaMemsetAsync(P[p].storage.ring, 0, 3 * lvl, s));
    if (P[p].grid.absorbing == NW_ABS_PML) NW_CUDA(cudaMemsetAsync(P[p].storage.pml_psi, 0, 4 * lvl, s));
  }
  for (int k = 0; k < Nmax; ++k) {
    const int na = batch_active(P, n, k, false);
    if (k % K == 0)
      for (int p = 0; p < na; ++p) {
        const bool pml = P[p].grid.absorbing == NW_ABS_PML;
        T* faces[2];
        if (pml) batch_pml_faces<T>(P[p], k, faces);
        int rc = snap_store<T>(&P[p].grid, &P[p].storage, P[p].acq.n_shots, ring_level<T>(P[p], k - 1),
                               ring_level<T>(P[p], k), k / K, s, pml ? faces : nullptr);
        if (rc) return rc;
      }
    bool any_pml = false;
    for (int p = 0; p < na; ++p) any_pml |= P[p].grid.absorbing == NW_ABS_PML;
    int rc = fork_join(
        s, any_pml,
        [&](cudaStream_t t) -> int {  // PML problems: receivers of level k and the layer cells
          for (int p = 0; p < na; ++p) {
            const nw_batch_problem& q = P[p];
            if (q.grid.absorbing != NW_ABS_PML) continue;
            int r = NW_OK;
            if (k % q.time.substeps == 0)
              r = launch_sample<T>(&q.grid, &q.acq, q.time.n_t, ring_level<T>(q, k), k / q.time.substeps,
                                   (T*)q.traces, t);
            if (!r) r = batch_pml_forward<T>(q, tu, k, false, t);
            if (r) return r;
          }
          return NW_OK;
        },
        [&](cudaStream_t t) -> int { return NW_DISPATCH_BATCH(launch_fwd_batch, T, tu.fwd, R, table, n, na, cta[na], k, 0, K, t); });
    if (rc) return rc;
    for (int p = 0; p < na; ++p) {  // the final receiver sample of problems ending after step k
      const nw_batch_problem& q = P[p];
      if (q.time.n_steps == k + 1 && q.time.n_steps % q.time.substeps == 0) {
        rc = launch_sample<T>(&q.grid, &q.acq, q.time.n_t, ring_level<T>(q, k + 1), (k + 1) / q.time.substeps,
                              (T*)q.traces, s);
        if (rc) return rc;
      }
    }
  }
  return NW_OK;
}

template <typename T>
int batch_adjoint_impl(const nw_batch_problem* P, int n, const Tune& tu, const void* table, cudaStream_t s) {
  const int K = P[0].storage.segment, Nmax = P[0].time.n_steps, R = P[0].grid.radius;
  const std::vector<int> fcta = batch_ctas<T>(P, n, tu.fwd), acta = batch_ctas<T>(P, n, tu.adj);
  for (int p = 0; p < n; ++p) {
    const nw_batch_problem& q = P[p];
    const size_t lvl = (size_t)q.acq.n_shots * q.grid.field_elems * sizeof(T);
    NW_CUDA(cudaMemsetAsync(q.work, 0, work_levels(&q.grid) * lvl, s));
    NW_CUDA(cudaMemsetAsync(q.grad_acc, 0, (size_t)n_acc_fields(&q.grid, tu, q.acq.n_shots) * q.grid.field_elems * sizeof(T), s));
  }
  auto adj_step = [&](int step) -> int {
    const int na = batch_active(P, n, step, true);
    bool any_pml = false;
    for (int p = 0; p < na; ++p) any_pml |= P[p].grid.absorbing == NW_ABS_PML;
    int rc = fork_join(
        s, any_pml,
        [&](cudaStream_t t) -> int {  // PML problems: the layer cells
          for (int p = 0; p < na; ++p)
            if (P[p].grid.absorbing == NW_ABS_PML) {
              const int r = batch_pml_adjoint<T>(P[p], tu, step, t);
              if (r) return r;
            }
          return NW_OK;
        },
        [&](cudaStream_t t) -> int { return NW_DISPATCH_BATCH(launch_adj_batch, T, tu.adj, R, table, n, na, acta[na], step, 0, K, t); });
    for (int p = 0; p < na && !rc; ++p)  // and their cotangents, once both halves are done
      if (P[p].grid.absorbing == NW_ABS_PML) rc = batch_pml_inject<T>(P[p], tu, step, s);
    return rc;
  };
  int rc = adj_step(Nmax);  // problems with the largest step count start: q^N = A C R^T g_N
  if (rc) return rc;
  for (int seg = Nmax > 0 ? (Nmax - 1) / K : -1; seg >= 0; --seg) {
    const int n0 = seg * K, n1 = std::min(n0 + K, Nmax);
    const int na0 = batch_active(P, n, n0, false);
    for (int p = 0; p < na0; ++p) {  // decode the segment's snapshots into the rings (and faces)
      const bool pml = P[p].grid.absorbing == NW_ABS_PML;
      T* faces[2];
      if (pml) batch_pml_faces<T>(P[p], n0, faces);
      rc = snap_load<T>(&P[p].grid, &P[p].storage, P[p].acq.n_shots, seg, ring_level<T>(P[p], n0 - 1),
                        ring_level<T>(P[p], n0), s, pml ? faces : nullptr);
      if (rc) return rc;
    }
    for (int k = n0; k < n1; ++k) {  // recompute Lap p^k into the segment buffers
      const int na = batch_active(P, n, k, false);
      bool any_pml = false;
      for (int p = 0; p < na; ++p) any_pml |= P[p].grid.absorbing == NW_ABS_PML;
      rc = fork_join(
          s, any_pml,
          [&](cudaStream_t t) -> int {
            for (int p = 0; p < na; ++p)
              if (P[p].grid.absorbing == NW_ABS_PML) {
                const int r = batch_pml_forward<T>(P[p], tu, k, true, t);
                if (r) return r;
              }
            return NW_OK;
          },
          [&](cudaStream_t t) -> int { return NW_DISPATCH_BATCH(launch_fwd_batch, T, tu.fwd, R, table, n, na, fcta[na], k, 1, K, t); });
      if (rc) return rc;
    }
    for (int step = n1 - 1; step >= n0; --step) {
      rc = adj_step(step);
      if (rc) return rc;
    }
  }
  return NW_OK;
}

}  // namespace

extern "C" {

size_t nw_batch_table_bytes(int32_t n_problems) { return n_problems < 1 ? 0 : batch_layout(n_problems).bytes; }

int nw_batch_prepare(const nw_batch_problem* problems, int32_t n_problems, const nw_tuning* tune, void* table,
                     void* stream) {
  if (!problems || n_problems < 1 || !table) return fail(NW_ERR_ARG, "invalid batch arguments");
  Tune tu;
  int rc = check_grid(&problems[0].grid);
  if (rc) return rc;
  rc = resolve_tune(&problems[0].grid, tune, &tu);
  if (rc) return rc;
  tu.fwd.depth = 1;  // batched steps take one step per launch
  rc = check_batch(problems, n_problems, tu);
  if (rc) return rc;
  if (problems[0].grid.dtype == NW_F32)
    return batch_prepare_impl<float>(problems, n_problems, tu, table, (cudaStream_t)stream);
  return batch_prepare_impl<double>(problems, n_problems, tu, table, (cudaStream_t)stream);
}

int nw_batch_forward(const nw_batch_problem* problems, int32_t n_problems, const nw_tuning* tune,
                     const void* table, void* stream) {
  if (!problems || n_problems < 1 || !table) return fail(NW_ERR_ARG, "invalid batch arguments");
  Tune tu;
  int rc = check_grid(&problems[0].grid);
  if (rc) return rc;
  rc = resolve_tune(&problems[0].grid, tune, &tu);
  if (rc) return rc;
  tu.fwd.depth = 1;  // batched steps take one step per launch
  rc = check_batch(problems, n_problems, tu);
  if (rc) return rc;
  if (problems[0].grid.dtype == NW_F32)
    return batch_forward_impl<float>(problems, n_problems, tu, table, (cudaStream_t)stream);
  return batch_forward_impl<double>(problems, n_problems, tu, table, (cudaStream_t)stream);
}

int nw_batch_adjoint(const nw_batch_problem* problems, int32_t n_problems, const nw_tuning* tune,
                     const void* table, void* stream) {
  if (!problems || n_problems < 1 || !table) return fail(NW_ERR_ARG, "invalid batch arguments");
  Tune tu;
  int rc = check_grid(&problems[0].grid);
  if (rc) return rc;
  rc = resolve_tune(&problems[0].grid, tune, &tu);
  if (rc) return rc;
  tu.fwd.depth = 1;  // batched steps take one step per launch
  rc = check_batch(problems, n_problems, tu);
  if (rc) return rc;
  if (problems[0].grid.dtype == NW_F32)
    return batch_adjoint_impl<float>(problems, n_problems, tu, table, (cudaStream_t)stream);
  return batch_adjoint_impl<double>(problems, n_problems, tu, table, (cudaStream_t)stream);
}

}  // extern "C"

// =============================================================================================
// Dirichlet time reversal: the forward step loop with the receivers' cells overwritten after
// every step.
// =============================================================================================
namespace {

template <typename T>
int time_reversal_impl(const nw_grid* g, const nw_medium* m, const nw_acquisition* a, const nw_time* t,
                       const nw_storage* st, const Tune& tu, const int64_t* cells, int n_cells, const T* traces,
                       cudaStream_t s) {
  const long long LE = g->field_elems;
  const int N = t->n_steps, M = t->substeps, n_t = t->n_t;
  Ring<T> L;
  L.base = (T*)st->ring;
  L.level_elems = LE;
  L.levels = ring_levels(st);
  NW_CUDA(cudaMemsetAsync(st->ring, 0, L.levels * (size_t)LE * sizeof(T), s));
  if (g->absorbing == NW_ABS_PML) NW_CUDA(cudaMemsetAsync(st->pml_psi, 0, 4 * (size_t)LE * sizeof(T), s));
  const nw::KGrid<T> kg = kgrid<T>(g);
  auto impose = [&](int n) -> int {  // the traces at reversed time T - n dt on level n
    const double u = (n_t - 1) - (double)n / M;
    const int j0 = std::min(std::max((int)std::floor(u), 0), n_t - 1);
    const int j1 = std::min(j0 + 1, n_t - 1);
    const double w = u - j0;
    nw::dirichlet_kernel<T><<<(n_cells + 127) / 128, 128, 0, s>>>(L.at(n), cells, n_cells, traces, n_t, j0, j1,
                                                                 (T)(1.0 - w), (T)w);
    NW_LAUNCHED();
    return NW_OK;
  };
  int rc = impose(0);
  if (rc) return rc;
  for (int n = 0; n < N; ++n) {
    rc = forward_step<T>(g, kg, m, a, t, tu, L, n, nullptr, nullptr, s, (T*)st->pml_psi);
    if (rc) return rc;
    rc = impose(n + 1);
    if (rc) return rc;
  }
  return NW_OK;
}

}  // namespace

extern "C" int nw_time_reversal(const nw_grid* g, const nw_medium* m, const nw_acquisition* a, const nw_time* t,
                                const nw_storage* st, const nw_tuning* tune, const int64_t* cells, int32_t n_cells,
                                const void* traces, void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  Tune tu;
  rc = resolve_tune(g, tune, &tu);
  if (rc) return rc;
  rc = check_run(g, m, a, t, st, tu);
  if (rc) return rc;
  if (a->n_shots != 1 || a->has_source) return fail(NW_ERR_ARG, "time reversal runs one shot without sources");
  if (!st->ring || (g->absorbing == NW_ABS_PML && !st->pml_psi)) return fail(NW_ERR_ARG, "time reversal needs the ring (and pml_psi with a PML)");
  if (n_cells < 1 || !cells || !traces) return fail(NW_ERR_ARG, "time reversal needs receiver cells and traces");
  if (g->dtype == NW_F32)
    return time_reversal_impl<float>(g, m, a, t, st, tu, cells, n_cells, (const float*)traces, (cudaStream_t)stream);
  return time_reversal_impl<double>(g, m, a, t, st, tu, cells, n_cells, (const double*)traces, (cudaStream_t)stream);
}

// ------------------------------------------------------------------------------------------------
// trace misfit: band-limited residual, masked mean square, adjoint source
// ------------------------------------------------------------------------------------------------
namespace {

int smallest_5smooth(int n) {  // scipy.fft.next_fast_len(n, real=True): the next 2^a 3^b 5^c >= n
  for (int m = std::max(n, 1);; ++m) {
    int r = m;
    for (int p : {2, 3, 5})
      while (r % p == 0) r /= p;
    if (r == 1) return m;
  }
}

int filter_log2_len(int n_t) {
  int k = 6;
  while ((1LL << k) < 2LL * n_t) ++k;
  return k;
}

// In-place radix-2 complex FFT (forward, float64) of length 2^k: iterative, bit-reversed input order.
void host_fft(std::vector<double>& re, std::vector<double>& im) {
  const size_t L = re.size();
  for (size_t i = 1, j = 0; i < L; ++i) {
    size_t bit = L >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      std::swap(re[i], re[j]);
      std::swap(im[i], im[j]);
    }
  }
  for (size_t len = 2; len <= L; len <<= 1) {
    const size_t half = len >> 1;
    for (size_t k = 0; k < half; ++k) {
      const double a = -2.0 * M_PI * (double)k / (double)len;
      const double wr = std::cos(a), wi = std::sin(a);
      for (size_t b = 0; b < L; b += len) {
        const size_t i = b + k, j = i + half;
        const double xr = re[j] * wr - im[j] * wi, xi = re[j] * wi + im[j] * wr;
        re[j] = re[i] - xr;
        im[j] = im[i] - xi;
        re[i] += xr;
        im[i] += xi;
      }
    }
  }
}

// Hp[p] = H_L[bitrev(p)] / L for the reference's filter of `kind` on traces of n_t samples, float64.
int filter_response(int kind, int n_t, double dt, double f, double taper, std::vector<double>* out) {
  if (n_t < 1 || !(dt > 0.0) || !(f > 0.0)) return fail(NW_ERR_ARG, "filter response needs n_t >= 1, dt > 0, f > 0");
  if (n_t > 8192) return fail(NW_ERR_UNSUPPORTED, "filtered traces are limited to 8192 samples");
  if (kind != NW_FILTER_LOWPASS && kind != NW_FILTER_GAUSSIAN) return fail(NW_ERR_ARG, "unknown filter kind");
  if (kind == NW_FILTER_LOWPASS && !(taper >= 0.0 && taper <= 1.0)) return fail(NW_ERR_ARG, "taper must be in [0, 1]");
  // the reference's FFT length and half spectrum (losses.py:28-48; sensor.py:33-38)
  const int N = kind == NW_FILTER_LOWPASS ? smallest_5smooth(2 * n_t) : 2 * n_t;
  const int J = N / 2;
  std::vector<double> w(J + 1);
  const double f1 = (1.0 - taper) * f;
  for (int j = 0; j <= J; ++j) {
    const double fj = (double)j * (1.0 / ((double)N * dt));  // rfftfreq's own rounding: j * (1 / (N dt))
    if (kind == NW_FILTER_GAUSSIAN) {
      w[j] = std::exp(-0.5 * (fj / f) * (fj / f));
    } else {
      double v = 1.0;
      if (fj > f1 && fj < f) v = 0.5 * (1.0 + std::cos(M_PI * (fj - f1) / std::max(f - f1, 1e-30)));
      if (fj >= f) v = 0.0;
      w[j] = v;
    }
  }
  // impulse response h = irfft(w, N) at lags 0..n_t-1 (it is even: h[N - k] = h[k])
  std::vector<double> ct(N);
  for (int m = 0; m < N; ++m) ct[m] = std::cos(2.0 * M_PI * (double)m / (double)N);
  const int M = (N % 2 == 0) ? J - 1 : J;
  std::vector<double> h(n_t);
  for (int k = 0; k < n_t; ++k) {
    double acc = 0.0;
    long long idx = 0;
    for (int j = 1; j <= M; ++j) {
      idx += k;
      if (idx >= N) idx %= N;
      acc += w[j] * ct[idx];
    }
    double v = w[0] + 2.0 * acc;
    if (N % 2 == 0) v += w[J] * ((k & 1) ? -1.0 : 1.0);
    h[k] = v / (double)N;
  }
  // the same lags on a power-of-two circle, its spectrum (real: the response is even), bit-reversed
  const int k2 = filter_log2_len(n_t);
  const size_t L = (size_t)1 << k2;
  std::vector<double> re(L, 0.0), im(L, 0.0);
  re[0] = h[0];
  for (int k = 1; k < n_t; ++k) re[k] = re[L - k] = h[k];
  host_fft(re, im);
  out->assign(L, 0.0);
  for (size_t p = 0; p < L; ++p) {
    size_t r = 0;
    for (int b = 0; b < k2; ++b)
      if (p & ((size_t)1 << b)) r |= (size_t)1 << (k2 - 1 - b);
    (*out)[p] = re[r] / (double)L;
  }
  return NW_OK;
}

int check_traces(const nw_traces* t) {
  if (!t) return fail(NW_ERR_ARG, "traces descriptor is NULL");
  if (t->dtype != NW_F32 && t->dtype != NW_F64) return fail(NW_ERR_ARG, "dtype must be NW_F32 or NW_F64");
  if (t->n_t < 1 || t->n_traces < 0) return fail(NW_ERR_ARG, "traces need n_t >= 1 and n_traces >= 0");
  if (t->mask_per_sample != 0 && t->mask_per_sample != 1) return fail(NW_ERR_ARG, "mask_per_sample must be 0 or 1");
  return NW_OK;
}

int check_filter_len(const nw_traces* t) {
  const int want = filter_log2_len(t->n_t);
  if (t->log2_len != want) return fail(NW_ERR_ARG, "log2_len must be nw_filter_log2_len(n_t)");
  const int cap = t->dtype == NW_F32 ? 14 : 13;
  if (t->log2_len > cap)
    return fail(NW_ERR_UNSUPPORTED, t->dtype == NW_F32 ? "filtered traces are limited to 8192 samples in float32"
                                                       : "filtered traces are limited to 4096 samples in float64");
  return NW_OK;
}

template <typename T>
int run_misfit_program(const nw_traces* t, nw::MisfitArgs<T> a, cudaStream_t s, int* ctas) {
  a.n_traces = t->n_traces;
  a.n_t = t->n_t;
  a.mask = (const T*)t->mask;
  a.mask_per_sample = t->mask_per_sample;
  int n_ctas = 1;
  if (a.n_filters == 0) {
    const long long N = t->n_traces * (long long)t->n_t;
    n_ctas = (int)std::max(1LL, std::min<long long>(nw::kMisfitCtas, (N + 255) / 256));
    if (N > 0) {
      nw::misfit_plain_kernel<T><<<n_ctas, 256, 0, s>>>(a);
      NW_LAUNCHED();
    } else if (a.partials) {
      NW_CUDA(cudaMemsetAsync(a.partials, 0, 2 * sizeof(double), s));
    }
    *ctas = n_ctas;
    return NW_OK;
  }
  const nw::fft::Groups G = nw::fft::make_groups(t->log2_len);
  const int L = 1 << t->log2_len;
  const size_t smem = (size_t)(G.tab_len + nw::fft::slot(L - 1) + 1) * sizeof(typename nw::fft::Cx<T>::t);
  const int threads = std::min(nw::misfit_threads<T>(), std::max(32, L >> 4));
  auto kern = nw::misfit_fft_kernel<T>;
  NW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, sms = 0, per_sm = 0;
  NW_CUDA(cudaGetDevice(&dev));
  NW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  NW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
  const long long pairs = (t->n_traces + 1) / 2;
  n_ctas = (int)std::max(1LL, std::min<long long>({(long long)nw::kMisfitCtas, pairs,
                                                   (long long)std::max(1, per_sm) * sms}));
  if (pairs > 0) {
    kern<<<n_ctas, threads, smem, s>>>(a, G);
    NW_LAUNCHED();
  } else if (a.partials) {
    NW_CUDA(cudaMemsetAsync(a.partials, 0, 2 * sizeof(double), s));
  }
  *ctas = n_ctas;
  return NW_OK;
}

template <typename T>
int misfit_prepare_impl(const nw_traces* t, const void* obs, const void* loss_response, int relative, double* state,
                        cudaStream_t s) {
  nw::MisfitArgs<T> a{};
  a.obs = (const T*)obs;
  a.partials = state;
  a.state = nullptr;
  const bool filtered = relative && loss_response;
  a.n_filters = filtered ? 1 : 0;
  if (filtered) {
    a.spec[0] = (const T*)loss_response;
    a.op[0] = nw::MF_LOAD_OBS;
    a.op[1] = nw::MF_LOSS | nw::MF_END;
  } else {
    a.op[0] = nw::MF_LOAD_OBS | nw::MF_LOSS;
  }
  int n_ctas = 0;
  const int rc = run_misfit_program<T>(t, a, s, &n_ctas);
  if (rc) return rc;
  const double count = t->mask ? 0.0 : (double)t->n_traces * (double)t->n_t;
  nw::misfit_finalize_kernel<<<1, 32, 0, s>>>(state, n_ctas, 1, relative ? 1 : 0, count);
  NW_LAUNCHED();
  return NW_OK;
}

template <typename T>
int misfit_impl(const nw_traces* t, const void* pred, const void* obs, const void* sensor, const void* loss,
                double* state, void* grad, cudaStream_t s) {
  nw::MisfitArgs<T> a{};
  a.pred = (const T*)pred;
  a.obs = (const T*)obs;
  a.grad = (T*)grad;
  a.state = state;
  a.partials = state;
  const unsigned store = grad ? nw::MF_STORE : nw::MF_END;
  int f = 0;
  if (sensor) {  // r = G pred - obs
    a.spec[f++] = (const T*)sensor;
    a.op[0] = nw::MF_LOAD_PRED;
    a.op[1] = nw::MF_SUB_OBS;
  } else {
    a.op[0] = nw::MF_LOAD_PRED | nw::MF_SUB_OBS;
  }
  if (loss) {
    a.spec[f++] = (const T*)loss;  // r_f = W r; sum m r_f^2; x = m r_f
    a.op[f] |= nw::MF_LOSS;
    if (grad) {
      a.spec[f++] = (const T*)loss;  // W^T = W
    }
  } else {
    a.op[f] |= nw::MF_LOSS;
  }
  if (sensor && grad) a.spec[f++] = (const T*)sensor;  // G^T = G
  a.n_filters = f;
  a.op[f] |= store;
  int n_ctas = 0;
  const int rc = run_misfit_program<T>(t, a, s, &n_ctas);
  if (rc) return rc;
  nw::misfit_finalize_kernel<<<1, 32, 0, s>>>(state, n_ctas, 0, 0, 0.0);
  NW_LAUNCHED();
  return NW_OK;
}

template <typename T>
int filter_impl(const nw_traces* t, const void* x, const void* response, void* y, cudaStream_t s) {
  nw::MisfitArgs<T> a{};
  a.pred = (const T*)x;
  a.grad = (T*)y;
  a.spec[0] = (const T*)response;
  a.n_filters = 1;
  a.op[0] = nw::MF_LOAD_PRED;
  a.op[1] = nw::MF_STORE;
  int n_ctas = 0;
  return run_misfit_program<T>(t, a, s, &n_ctas);
}

}  // namespace

extern "C" int nw_filter_log2_len(int32_t n_t) { return n_t < 1 ? fail(NW_ERR_ARG, "n_t must be >= 1") : filter_log2_len(n_t); }

extern "C" int nw_filter_response(int32_t kind, int32_t n_t, double dt, double f, double taper, int32_t dtype,
                                  void* out) {
  if (!out) return fail(NW_ERR_ARG, "out is NULL");
  if (dtype != NW_F32 && dtype != NW_F64) return fail(NW_ERR_ARG, "dtype must be NW_F32 or NW_F64");
  std::vector<double> hp;
  const int rc = filter_response(kind, n_t, dt, f, taper, &hp);
  if (rc) return rc;
  for (size_t i = 0; i < hp.size(); ++i) {
    if (dtype == NW_F32) ((float*)out)[i] = (float)hp[i];
    else ((double*)out)[i] = hp[i];
  }
  return NW_OK;
}

extern "C" int nw_trace_filter(const nw_traces* t, const void* x, const void* response, void* y, void* stream) {
  int rc = check_traces(t);
  if (rc) return rc;
  if (!x || !response || !y) return fail(NW_ERR_ARG, "trace filter needs x, response and y");
  rc = check_filter_len(t);
  if (rc) return rc;
  if (t->dtype == NW_F32) return filter_impl<float>(t, x, response, y, (cudaStream_t)stream);
  return filter_impl<double>(t, x, response, y, (cudaStream_t)stream);
}

extern "C" int nw_misfit_prepare(const nw_traces* t, const void* obs, const void* loss_response, int32_t relative,
                                 double* state, void* stream) {
  int rc = check_traces(t);
  if (rc) return rc;
  if (!obs || !state) return fail(NW_ERR_ARG, "misfit prepare needs obs and state");
  if (relative && loss_response) {
    rc = check_filter_len(t);
    if (rc) return rc;
  }
  if (t->dtype == NW_F32)
    return misfit_prepare_impl<float>(t, obs, loss_response, relative, state, (cudaStream_t)stream);
  return misfit_prepare_impl<double>(t, obs, loss_response, relative, state, (cudaStream_t)stream);
}

extern "C" int nw_misfit(const nw_traces* t, const void* pred, const void* obs, const void* sensor_response,
                         const void* loss_response, double* state, void* grad, void* stream) {
  int rc = check_traces(t);
  if (rc) return rc;
  if (!pred || !obs || !state) return fail(NW_ERR_ARG, "misfit needs pred, obs and state");
  if (sensor_response || loss_response) {
    rc = check_filter_len(t);
    if (rc) return rc;
  }
  if (t->dtype == NW_F32)
    return misfit_impl<float>(t, pred, obs, sensor_response, loss_response, state, grad, (cudaStream_t)stream);
  return misfit_impl<double>(t, pred, obs, sensor_response, loss_response, state, grad, (cudaStream_t)stream);
}
