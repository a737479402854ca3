// Host side of libafid_gpu: contexts, boxes, metric tables, batches, launch
// sequences and the C-ABI of include/afid_gpu.h.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "afid_device.cuh"
#include "k_fft.cuh"
#include "k_fftw.cuh"
#include "k_routine.cuh"
#include "k_stencil.cuh"
#include "../../include/afid_gpu.h"

using namespace afid;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(call)                                                                            \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail(AFID_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#define CKL()                                                                               \
  do {                                                                                      \
    cudaError_t e_ = cudaGetLastError();                                                    \
    if (e_ != cudaSuccess)                                                                  \
      return fail(AFID_ECUDA, "launch: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

// Launch families; each has its own table of tile offsets per batch.  The
// y transforms of boxes with a warp plan run in FAM_WY8/12 (values per
// lane), the others in FAM_FY; likewise the z transforms in FAM_WZ8/12 and
// FAM_FZ.
enum Fam { FAM_K1 = 0, FAM_COL, FAM_CELL, FAM_DIAG, FAM_FY, FAM_FZ, FAM_PX, FAM_K2,
           FAM_WY8, FAM_WY12, FAM_WZ8, FAM_WZ12, NFAM };
constexpr int WY_NV = 2;
constexpr int WY_V[WY_NV] = {8, 12};
constexpr int HIST_CAP = 4096;

struct HostBox {
  int id = -1;
  afid_box_params prm{};
  BoxDev dev{};           // descriptor with device pointers
  BoxDev *d_self = nullptr;  // device copy of dev (active = 1), for single-box kernels
  void *mem_fields = nullptr, *mem_scratch = nullptr, *mem_small = nullptr, *mem_routine = nullptr;
  size_t scratch_doubles = 0;
  std::vector<double> xc;                // node positions (host copy, for the output diagnostics)
  double *d_out = nullptr;               // device staging of the output diagnostics (grown on demand)
  size_t out_doubles = 0;
  std::vector<double> stats;             // AFID_NSTAT x nxm accumulators (stat_arrays)
  int nstatsamples = 0;
};

struct Batch {
  std::vector<int> ids;
  BoxDev *d_boxes = nullptr;
  int *d_off = nullptr;     // NFAM x (nbox + 1)
  int total[NFAM] = {};
  size_t smem_y = 0, smem_z = 0;
  FftSmem sm_y{0, 0}, sm_z{0, 0};   // slot and twiddle sizes of the persistent transforms
  int grid_y = 0, grid_z = 0;       // their resident grids
  int k2_block = 256;               // threads per block of the back-substitution kernel
  size_t smem_wy[WY_NV] = {};       // shared memory and resident grids of the warp y transforms
  int grid_wy[WY_NV] = {};
  int grid_wz[WY_NV] = {};          // resident grids of the warp z transforms (shared memory as y)
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t gstream = nullptr;
  int graph_kernels = 0;    // kernel nodes of the captured step graph
  int k1_minb = 4;          // variant of the explicit/forward kernel (tuning, K1_VMIN..K1_VMAX)
  // A large set is stepped through its graph as two halves of about equal
  // cells, each with its own graph on its own stream: the halves drift
  // apart, so that one half's latency-bound transforms run beside the other
  // half's bandwidth-bound stencils.  The halves are batches of their own
  // (looked up by their ids, never split again).
  bool split = false;
  std::vector<int> half_ids[2];
};

// splitting rule of afid_step_graph: sets of at least this many boxes and
// cells run as two halves (afid_ctx_set_split_sets turns it off)
constexpr int SPLIT_MIN_BOXES = 8;
constexpr long long SPLIT_MIN_CELLS = 4LL << 20;

long long cdiv(long long a, long long b) { return (a + b - 1) / b; }

// FFT plan of length n: radix 16 for every four factors of two, one radix
// 8, 4 or 2 for the rest, then 3, 5 and 7.  The power-of-two passes come
// first, so that the stride Ns of every pass but those after a second odd
// radix is a power of two (shift and mask indexing).
int factor_radices(int n, int *rad, int *np) {
  int m = n, a = 0, c = 0;
  while (m % 2 == 0) { m /= 2; ++a; }
  int tmp[16];
  while (a >= 4 && c < 15) { tmp[c++] = 16; a -= 4; }
  if (a == 3) tmp[c++] = 8; else if (a == 2) tmp[c++] = 4; else if (a == 1) tmp[c++] = 2;
  const int odd[3] = {3, 5, 7};
  for (int q = 0; q < 3; ++q)
    while (m % odd[q] == 0 && c < 15) { tmp[c++] = odd[q]; m /= odd[q]; }
  if (m != 1 || c > 15 || c == 0) return -1;
  for (int x = 0; x < c; ++x) rad[x] = tmp[x];
  rad[c] = 0;
  *np = c;
  return 0;
}

// Warp plan of an n-point transform (k_fftw.cuh): V values per lane (8 or
// 12; 16 and 24 spilled registers at two blocks per SM), G = n / V lanes per
// line (a power of two, min_g <= G <= 32), and a radix sequence whose
// radices all divide V, power-of-two radices first; the fewest passes win,
// then the fewer values per lane.  The y transforms need min_g = 2: their
// staged rows (2 LPW rows of N + 2 doubles, or of N/2 + 1 complex values)
// fit a warp buffer only with LPW = 32 / G <= 16.  Returns 0 (no plan) for
// sizes the tile kernels keep: lines longer than WARP_PLAN_MAX_N, where the
// tile kernels measured faster (384 and 768 points).
constexpr int WARP_PLAN_MAX_N = WF_MAX_N;
int warp_plan(int n, int *v_out, int *g_out, int *rad, int *np, int min_g = 1) {
  static const int cand[7] = {16, 12, 8, 6, 4, 3, 2};
  if (n > WARP_PLAN_MAX_N) return 0;
  int best_v = 0, best_np = 99, best[8] = {};
  for (int vi = 0; vi < WY_NV; ++vi) {
    const int V = WY_V[vi];
    if (n % V) continue;
    const int G = n / V;
    if (G < min_g || G > 32 || (G & (G - 1))) continue;
    // depth-first search for the shortest factorisation into radices dividing V
    int cur[8], found[8] = {}, found_np = 99;
    std::function<void(int, int)> dfs = [&](int m, int d) {
      if (d >= found_np || d >= 8) return;
      if (m == 1) {
        found_np = d;
        for (int q = 0; q < d; ++q) found[q] = cur[q];
        return;
      }
      for (int c : cand)
        if (V % c == 0 && m % c == 0) {
          cur[d] = c;
          dfs(m / c, d + 1);
        }
    };
    dfs(n, 0);
    if (found_np < best_np) {
      best_np = found_np;
      best_v = V;
      for (int q = 0; q < found_np; ++q) best[q] = found[q];
    }
  }
  if (!best_v) return 0;
  // power-of-two radices first (shift-and-mask indexing of the strides)
  int o = 0;
  for (int q = 0; q < best_np; ++q) if ((best[q] & (best[q] - 1)) == 0) rad[o++] = best[q];
  for (int q = 0; q < best_np; ++q) if ((best[q] & (best[q] - 1)) != 0) rad[o++] = best[q];
  *v_out = best_v;
  *g_out = n / best_v;
  *np = best_np;
  return 1;
}

// Variants of the explicit/forward kernel: tile height TI (block of 32 TI
// threads), resident blocks per SM and planes per barrier.
//   2: 32x8 tiles, 2 blocks/SM        3: 32x8 tiles, 3 blocks/SM (80 registers)
//   4: 32x8 tiles, two planes per barrier (a 7-plane ring of 150 KB: one
//      block per SM at 128 registers)
//   5: 32x4 tiles, 4 blocks/SM        6: 32x2 tiles, 8 blocks/SM
//   7: 32x4 tiles, 5 blocks/SM        8: 32x4 tiles, 6 blocks/SM
constexpr int K1_VMIN = 2, K1_VMAX = 8;
constexpr int K1_DEFAULT = 4;   // the variant the tuner picks for the large boxes (768^2, 1280^2)
int k1_tile_height(int variant) { return (variant == 5 || variant >= 7) ? 4 : variant == 6 ? 2 : 8; }

long long tiles_of(const BoxDev &B, int fam, int k1_variant = 2, int k2_block = 256) {
  switch (fam) {
    case FAM_K2: return cdiv(B.plane, k2_block);
    case FAM_K1: return cdiv(B.nym, K1_TJ) * cdiv(B.nzm, k1_tile_height(k1_variant));
    case FAM_COL: return cdiv(B.plane, 256);
    case FAM_CELL: return cdiv((long long)B.nxm * B.plane, 256);
    case FAM_DIAG: return cdiv(B.plane, 256);
    case FAM_FY: return B.wy_v ? 0 : (long long)B.nxm * cdiv(B.nzm, 2 * fft_y_pairs(B));
    case FAM_WY8: case FAM_WY12:
      return B.wy_v == WY_V[fam - FAM_WY8] ? (long long)B.nxm * wy_units_per_plane(B) : 0;
    case FAM_FZ: return B.wz_v ? 0 : (long long)B.nxm * cdiv(B.nymh, fft_z_lines(B));
    case FAM_WZ8: case FAM_WZ12:
      return B.wz_v == WY_V[fam - FAM_WZ8] ? (long long)B.nxm * wz_units_per_plane(B) : 0;
    case FAM_PX: return cdiv(px_pairs(B.nzm, B.nymh), 256);
  }
  return 0;
}

struct Sizes {
  long long nx, plane, fsize, nspec, npiv, scratch, small;
};

Sizes sizes_of(const afid_box_params &p) {
  Sizes s;
  s.nx = p.nxm + 1;
  s.plane = (long long)p.nym * p.nzm;
  s.fsize = s.nx * s.plane;
  s.nspec = (long long)p.nxm * p.nzm * (p.nym / 2 + 1);
  s.npiv = (long long)p.nxm * px_pairs(p.nzm, p.nym / 2 + 1);   // pivot table: kz <= nzm/2
  long long pois = 3 * s.nspec + 1 + (long long)p.nxm * s.plane;   // dph 16-byte aligned
  s.scratch = pois > 4 * s.fsize ? pois : 4 * s.fsize;
  // tables + twiddles + coef + nu partials + history + scalars (in doubles)
  s.small = (long long)T_NK * s.nx + p.nzm + p.nym + 2LL * (p.nym + p.nzm) +
            (long long)SYS_N * C_N * s.nx + 2 * NU_BLOCKS + (long long)HIST_CAP * HIST_FIELDS +
            (long long)(sizeof(BoxScalars) / 8 + 8) + s.plane +
            64;   // alignment of the scalars and the 128-byte TMA map (64-byte aligned)
  return s;
}

// ---- metric tables: CreateGrid.F90:129-266 and InitPressureSolver.F90:22-59
void build_tables(const afid_box_params &p, const double *xc, std::vector<double> &tab) {
  const int nxm = p.nxm, nym = p.nym, nzm = p.nzm, nx = nxm + 1;
  tab.assign((size_t)T_NK * nx + nzm + nym, 0.0);
  auto T = [&](int t, int k) -> double & { return tab[(size_t)t * nx + k]; };
  const double pi = 2.0 * std::asin(1.0);
  const double dx = (double)nxm / p.alx3;
  const double dxq = dx * dx;
  std::vector<double> g3rm(nx, 0.0), g3rc(nx, 0.0);
  for (int kc = 1; kc <= nxm; ++kc) g3rm[kc - 1] = (xc[kc] - xc[kc - 1]) * dx;
  for (int kc = 2; kc <= nxm; ++kc) g3rc[kc - 1] = (xc[kc] - xc[kc - 2]) * dx * 0.5;
  g3rc[0] = (xc[1] - xc[0]) * dx;
  g3rc[nx - 1] = (xc[nx - 1] - xc[nxm - 1]) * dx;
  for (int kc = 1; kc <= nxm; ++kc) {
    T(T_UDX3M, kc - 1) = dx / g3rm[kc - 1];
    T(T_UDX3C, kc - 1) = dx / g3rc[kc - 1];
  }
  T(T_UDX3C, nx - 1) = dx / g3rc[nx - 1];
  // centred second derivative
  T(T_AC3CK, 0) = 1.0; T(T_AC3CK, nx - 1) = 1.0;
  for (int kc = 2; kc <= nxm; ++kc) {
    const double a33 = dxq / g3rc[kc - 1];
    const double a33p = 1.0 / g3rm[kc - 1];
    const double a33m = 1.0 / g3rm[kc - 2];
    T(T_AP3CK, kc - 1) = a33 * a33p;
    T(T_AM3CK, kc - 1) = a33 * a33m;
    T(T_AC3CK, kc - 1) = -(T(T_AP3CK, kc - 1) + T(T_AM3CK, kc - 1));
  }
  // staggered, with the wall conditions
  for (int kc = 2; kc <= nxm - 1; ++kc) {
    const double a33 = dxq / g3rm[kc - 1];
    const double a33p = +a33 / g3rc[kc];
    const double a33m = +a33 / g3rc[kc - 1];
    T(T_AP3SK, kc - 1) = a33p;
    T(T_AM3SK, kc - 1) = a33m;
    T(T_AC3SK, kc - 1) = -(T(T_AP3SK, kc - 1) + T(T_AM3SK, kc - 1));
  }
  {
    const int kc = 1;
    const double a33 = dxq / g3rm[kc - 1];
    const double a33p = +a33 / g3rc[kc];
    const double a33m = +a33 / g3rc[kc - 1];
    T(T_AP3SK, kc - 1) = a33p;
    T(T_AM3SK, kc - 1) = 0.0;
    T(T_AC3SK, kc - 1) = -(a33p + p.inslws * a33m * 2.0);
  }
  {
    const int kc = nxm;
    const double a33 = dxq / g3rm[kc - 1];
    const double a33p = +a33 / g3rc[kc];
    const double a33m = +a33 / g3rc[kc - 1];
    T(T_AM3SK, kc - 1) = a33m;
    T(T_AP3SK, kc - 1) = 0.0;
    T(T_AC3SK, kc - 1) = -(a33m + p.inslwn * a33p * 2.0);
  }
  // temperature
  T(T_AC3SSK, 0) = 1.0;
  for (int kc = 2; kc <= nxm; ++kc) {
    const double a33 = dxq / g3rc[kc - 1];
    const double a33p = 1.0 / g3rm[kc - 1];
    const double a33m = 1.0 / g3rm[kc - 2];
    T(T_AP3SSK, kc - 1) = a33 * a33p;
    T(T_AM3SSK, kc - 1) = a33 * a33m;
    T(T_AC3SSK, kc - 1) = -(T(T_AP3SSK, kc - 1) + T(T_AM3SSK, kc - 1));
  }
  T(T_AC3SSK, nx - 1) = 1.0;
  // Poisson x-coefficients (kmc(1) = 0, kpc(nxm) = 0)
  for (int kc = 1; kc <= nxm; ++kc) {
    const int kp = (kc == nxm) ? kc : kc + 1;
    const double kmc = (kc == 1) ? 0.0 : 1.0;
    const double kpc = (kc == nxm) ? 0.0 : 1.0;
    const double a33icc = kmc * dxq / g3rc[kc - 1];
    const double a33icp = kpc * dxq / g3rc[kp - 1];
    const double ugmmm = 1.0 / g3rm[kc - 1];
    T(T_AMPHK, kc - 1) = a33icc * ugmmm;
    T(T_APPHK, kc - 1) = a33icp * ugmmm;
    T(T_ACPHK, kc - 1) = -(T(T_AMPHK, kc - 1) + T(T_APPHK, kc - 1));
  }
  for (int k = 0; k < nx; ++k) { T(T_XC, k) = xc[k]; T(T_G3RC, k) = g3rc[k]; T(T_G3RM, k) = g3rm[k]; }
  // modified wavenumbers
  double *ak1 = &tab[(size_t)T_NK * nx];
  double *ak2 = ak1 + nzm;
  const int nzmh = nzm / 2 + 1, nymh = nym / 2 + 1;
  for (int i = 1; i <= nzm; ++i) {
    const double ao = (i <= nzmh) ? (i - 1) * 2.0 * pi : -(nzm - i + 1) * 2.0 * pi;
    const double f = (double)nzm / p.zlen;
    ak1[i - 1] = 2.0 * (1.0 - std::cos(ao / nzm)) * (f * f);
  }
  for (int j = 1; j <= nym; ++j) {
    const double ap = (j <= nymh) ? (j - 1) * 2.0 * pi : -(nym - j + 1) * 2.0 * pi;
    const double f = (double)nym / p.ylen;
    ak2[j - 1] = 2.0 * (1.0 - std::cos(ap / nym)) * (f * f);
  }
}

void build_twiddles(int n, double2 *w) {
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < n; ++k) {
    const long double a = 2.0L * pi * (long double)k / (long double)n;
    w[k] = make_double2((double)cosl(a), (double)(-sinl(a)));
  }
}


// ---- TMA maps -----------------------------------------------------------------
// cuTensorMapEncodeTiled is a driver entry point; it is looked up through the
// runtime so that the library needs no link-time dependency on libcuda.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// largest divisor of n not above 256 (kz rows per TMA box)
int tma_rows(int n) {
  for (int r = n < 256 ? n : 256; r > 1; --r)
    if (n % r == 0) return r;
  return 1;
}

// encode the z-transform map of box d (its spec array, box 2L x rb doubles)
int encode_z_map(BoxDev &d, CUtensorMap *out) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return fail(AFID_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const int L = fft_z_lines(d);
  d.fz_rb = tma_rows(d.nzm);
  const cuuint64_t dims[2] = {(cuuint64_t)2 * d.nymh, (cuuint64_t)d.nxm * d.nzm};
  const cuuint64_t strides[1] = {(cuuint64_t)2 * d.nymh * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * L), (cuuint32_t)d.fz_rb};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void *)d.spec, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(AFID_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return 0;
}

// encode box d's z map and copy it to its device slot d.tm_z
int write_z_map(BoxDev &d, cudaStream_t st) {
  CUtensorMap m;
  int rc = encode_z_map(d, &m);
  if (rc) return rc;
  CK(cudaMemcpyAsync((void *)d.tm_z, &m, sizeof m, cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  return 0;
}

}  // namespace

struct afid_ctx {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  std::map<int, HostBox *> boxes;
  int next_id = 0;
  std::map<std::vector<int>, Batch *> batches;
  std::vector<double> staging_host;
  // streams and events of split batches (created on first use); split_sets
  // 0 keeps every set whole (afid_ctx_set_split_sets)
  int split_sets = 1;
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
  // staging of afid_boxes_get_scalars: device and pinned host records
  // (one per stream the context has used, so that calls on different
  // streams never share a staging array)
  struct RecStage {
    BoxScalars *d = nullptr, *h = nullptr;
    int n = 0;     // records of BoxScalars size it holds
  };
  std::map<cudaStream_t, RecStage> rec_stage;
};

namespace {

int set_device(afid_ctx *c) {
  CK(cudaSetDevice(c->device));
  return 0;
}

void free_batch(Batch *bt) {
  if (!bt) return;
  if (bt->gexec) cudaGraphExecDestroy(bt->gexec);
  if (bt->d_boxes) cudaFree(bt->d_boxes);
  if (bt->d_off) cudaFree(bt->d_off);
  delete bt;
}

int get_box(afid_ctx *c, int id, HostBox **out) {
  auto it = c->boxes.find(id);
  if (it == c->boxes.end()) return fail(AFID_ENOBOX, "unknown box id %d", id);
  *out = it->second;
  return 0;
}

int init_kernel_attrs();
int wy_shapes(const std::vector<BoxDev> &devs, const int *total, size_t *smem, int *grid, int *grid_z);


// slot sizes (complex values) and twiddle lengths of the persistent
// transforms, grown to cover box d (the directions d runs in a tile kernel)
void fft_smem_grow(const BoxDev &d, FftSmem &y, FftSmem &z, int &twy, int &twz) {
  if (!d.wy_v) {
    y.slot = std::max(y.slot, fft_y_slot(d.nym, fft_y_pairs(d)));
    y.tw = std::max(y.tw, d.nym);
    twy = std::max(twy, d.nym);
  }
  if (!d.wz_v) {
    z.slot = std::max(z.slot, fft_z_lines(d) * d.nzm);
    z.tw = std::max(z.tw, d.nzm);
    twz = std::max(twz, d.nzm);
  }
}

// resident grid of a persistent transform: SMs x blocks per SM, at most tiles
template <class K>
int fft_grid(K kernel, size_t smem, int tiles, int *grid) {
  int dev = 0, nsm = 0, occ = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, FFT_T, smem));
  if (occ < 1) return fail(AFID_ESIZE, "transform block of %zu bytes of shared memory does not fit an SM", smem);
  *grid = std::max(1, std::min(tiles, nsm * occ));
  return 0;
}

// Block size of the back-substitution kernel.  Each of its threads marches
// a whole column, so the grid runs in waves of (SMs x resident threads)
// columns and a last, partly filled wave costs a full column march.  Of the
// block sizes that keep the SMs' thread slots filled, pick the one whose
// waves are filled best (ties: more resident threads).
int k2_block_size(const std::vector<BoxDev> &devs, int *out) {
  int dev = 0, nsm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  double best = 1e30;
  int best_res = 0;
  *out = 256;
  for (int bs = 128; bs <= 256; bs += 32) {
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_implicit_bwd, bs, 0));
    if (occ < 1) continue;
    const long long res = (long long)nsm * occ * bs;   // resident threads
    long long cols = 0;
    for (const BoxDev &d : devs) cols += cdiv(d.plane, bs) * bs;
    const double waves = (double)cols / (double)res;
    const double cost = std::ceil(waves) / waves;   // >= 1: time over the ideal
    if (cost < best - 1e-9 || (cost < best + 1e-9 && res > best_res)) {
      best = cost;
      best_res = (int)(res / nsm);
      *out = bs;
    }
  }
  return 0;
}

int get_batch(afid_ctx *c, const int *ids, int n, Batch **out, bool allow_split = true) {
  if (n <= 0 || !ids) return fail(AFID_EINVAL, "empty box set");
  std::vector<int> key(ids, ids + n);
  auto it = c->batches.find(key);
  if (it != c->batches.end()) { *out = it->second; return 0; }
  std::vector<BoxDev> devs;
  std::vector<int> off((size_t)NFAM * (n + 1), 0);
  Batch *bt = new Batch();
  int twy_max = 0, twz_max = 0;
  bt->ids = key;
  for (int b = 0; b < n; ++b) {
    HostBox *hb;
    int rc = get_box(c, ids[b], &hb);
    if (rc) { delete bt; return rc; }
    BoxDev d = hb->dev;
    d.active = 1;
    devs.push_back(d);
    fft_smem_grow(d, bt->sm_y, bt->sm_z, twy_max, twz_max);
  }
  // Boxes of more planes first: a block of a column march (or of the
  // explicit kernel's tiles) takes time in proportion to its box's nxm, and
  // with the longest blocks started first the short ones fill the end of the
  // launch.  pos[b] is the caller's position of the batch's box b.
  std::vector<int> pos(n), bids(n);
  for (int b = 0; b < n; ++b) pos[b] = b;
  std::stable_sort(pos.begin(), pos.end(), [&](int a, int b) { return devs[a].nxm > devs[b].nxm; });
  {
    std::vector<BoxDev> sorted(n);
    for (int b = 0; b < n; ++b) { sorted[b] = devs[pos[b]]; bids[b] = ids[pos[b]]; }
    devs.swap(sorted);
  }
  bt->smem_y = (size_t)(2 * bt->sm_y.slot + twy_max) * 16 + FFT_TAIL_BYTES;   // + mbarriers, descriptor
  bt->smem_z = (size_t)(2 * bt->sm_z.slot + twz_max) * 16 + FFT_TAIL_BYTES;
  {
    // one variant of the explicit/forward kernel per launch: the one the
    // boxes holding most of the cells ask for
    long long w[K1_VMAX + 1] = {};
    for (const BoxDev &d : devs) w[d.k1_minb >= K1_VMIN && d.k1_minb <= K1_VMAX ? d.k1_minb : K1_DEFAULT] += d.fsize;
    bt->k1_minb = K1_DEFAULT;
    for (int v = K1_VMIN; v <= K1_VMAX; ++v)
      if (w[v] > w[bt->k1_minb]) bt->k1_minb = v;
    const char *e = getenv("AFID_K1_VARIANT");
    if (e && atoi(e) >= K1_VMIN && atoi(e) <= K1_VMAX) bt->k1_minb = atoi(e);
  }
  {
    int rc = k2_block_size(devs, &bt->k2_block);
    if (rc) { delete bt; return rc; }
  }
  for (int f = 0; f < NFAM; ++f) {
    long long acc = 0;
    for (int b = 0; b < n; ++b) {
      off[(size_t)f * (n + 1) + b] = (int)acc;
      acc += tiles_of(devs[b], f, bt->k1_minb, bt->k2_block);
    }
    if (acc > 0x7fffffffLL) { delete bt; return fail(AFID_ESIZE, "grid too large"); }
    off[(size_t)f * (n + 1) + n] = (int)acc;
    bt->total[f] = (int)acc;
  }
  off.insert(off.end(), pos.begin(), pos.end());   // the positions follow the tile tables
  if (cudaMalloc(&bt->d_boxes, sizeof(BoxDev) * n) != cudaSuccess ||
      cudaMalloc(&bt->d_off, sizeof(int) * off.size()) != cudaSuccess) {
    free_batch(bt);
    return fail(AFID_ENOMEM, "batch descriptor allocation failed");
  }
  CK(cudaMemcpy(bt->d_boxes, devs.data(), sizeof(BoxDev) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(bt->d_off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
  {
    int rc = init_kernel_attrs();
    if (!rc) rc = fft_grid(k_fft_y_fwd, bt->smem_y, bt->total[FAM_FY], &bt->grid_y);
    if (!rc) rc = fft_grid(k_fft_z<-1>, bt->smem_z, bt->total[FAM_FZ], &bt->grid_z);
    if (!rc) rc = wy_shapes(devs, bt->total, bt->smem_wy, bt->grid_wy, bt->grid_wz);
    if (rc) { free_batch(bt); return rc; }
  }
  if (allow_split && n >= SPLIT_MIN_BOXES) {
    long long cells = 0;
    for (const BoxDev &d : devs) cells += (long long)d.nxm * d.plane;
    if (cells >= SPLIT_MIN_CELLS) {
      // greedy balance of cells, largest boxes first; each half keeps the
      // set's order
      std::vector<int> order(n), side(n, 0);
      for (int b = 0; b < n; ++b) order[b] = b;
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (long long)devs[a].nxm * devs[a].plane > (long long)devs[b].nxm * devs[b].plane;
      });
      long long load[2] = {0, 0};
      for (int b : order) {
        const int h = load[1] < load[0] ? 1 : 0;
        side[b] = h;
        load[h] += (long long)devs[b].nxm * devs[b].plane;
      }
      for (int b = 0; b < n; ++b) bt->half_ids[side[b]].push_back(bids[b]);
      bt->split = !bt->half_ids[0].empty() && !bt->half_ids[1].empty();
    }
  }
  c->batches[key] = bt;
  *out = bt;
  return 0;
}

// Shared memory and resident grids (in blocks of wf_warps(V) warps, at
// most one warp per unit) of the warp y and z transforms of a set of boxes.
int wy_shapes(const std::vector<BoxDev> &devs, const int *total, size_t *smem, int *grid, int *grid_z) {
  (void)devs;
  int dev = 0, nsm = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  for (int c = 0; c < WY_NV; ++c) {
    smem[c] = wf_smem_bytes(WY_V[c]);
    grid[c] = grid_z[c] = 0;
    for (int zd = 0; zd < 2; ++zd) {
      const int units = total[(zd ? FAM_WZ8 : FAM_WY8) + c];
      if (!units) continue;
      int occ = 0;
      const int nt = 32 * wf_warps(WY_V[c]);
      if (c == 0 && !zd) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fftw_y_fwd<8>, nt, smem[c]));
      else if (!zd) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fftw_y_fwd<12>, nt, smem[c]));
      else if (c == 0) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fftw_z<-1, 8>, nt, smem[c]));
      else CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fftw_z<-1, 12>, nt, smem[c]));
      if (occ < 1) return fail(AFID_ESIZE, "warp transform block of %zu bytes does not fit an SM", smem[c]);
      (zd ? grid_z : grid)[c] = std::max(1, std::min((int)cdiv(units, wf_warps(WY_V[c])), nsm * occ));
    }
  }
  return 0;
}

// The z transforms of a batch (SGN -1 forward, +1 inverse): the tile kernel
// for boxes without a warp plan, one warp-kernel launch per class present.
template <int SGN, class BD>
int launch_fft_z(const int *total, BD bd, int grid_z, size_t smem_z, FftSmem sm_z, const int *grid_wz,
                 const size_t *smem_wy, cudaStream_t s, int ns) {
  if (total[FAM_FZ] > 0) {
    k_fft_z<SGN><<<grid_z, FFT_T, smem_z, s>>>(bd(FAM_FZ), ns, sm_z, total[FAM_FZ]);
    CKL();
  }
  for (int c = 0; c < WY_NV; ++c) {
    const int f = FAM_WZ8 + c;
    if (!total[f]) continue;
    if (c == 0) k_fftw_z<SGN, 8><<<grid_wz[c], 32 * wf_warps(8), smem_wy[c], s>>>(bd(f), ns, total[f]);
    else k_fftw_z<SGN, 12><<<grid_wz[c], 32 * wf_warps(12), smem_wy[c], s>>>(bd(f), ns, total[f]);
    CKL();
  }
  return 0;
}

// The y transforms of a batch: the tile kernel for boxes without a warp
// plan, one warp-kernel launch per values-per-lane class present.
template <class BD>
int launch_fft_y(bool fwd, const int *total, BD bd, int grid_y, size_t smem_y, FftSmem sm_y, const int *grid_wy,
                 const size_t *smem_wy, cudaStream_t s, int ns) {
  if (total[FAM_FY] > 0) {
    if (fwd) k_fft_y_fwd<<<grid_y, FFT_T, smem_y, s>>>(bd(FAM_FY), ns, sm_y, total[FAM_FY]);
    else k_fft_y_inv<<<grid_y, FFT_T, smem_y, s>>>(bd(FAM_FY), ns, sm_y, total[FAM_FY]);
    CKL();
  }
  for (int c = 0; c < WY_NV; ++c) {
    const int f = FAM_WY8 + c;
    if (!total[f]) continue;
    const BatchDev b = bd(f);
    if (c == 0) {
      if (fwd) k_fftw_y_fwd<8><<<grid_wy[c], 32 * wf_warps(8), smem_wy[c], s>>>(b, ns, total[f]);
      else k_fftw_y_inv<8><<<grid_wy[c], 32 * wf_warps(8), smem_wy[c], s>>>(b, ns, total[f]);
    } else {
      if (fwd) k_fftw_y_fwd<12><<<grid_wy[c], 32 * wf_warps(12), smem_wy[c], s>>>(b, ns, total[f]);
      else k_fftw_y_inv<12><<<grid_wy[c], 32 * wf_warps(12), smem_wy[c], s>>>(b, ns, total[f]);
    }
    CKL();
  }
  return 0;
}

// the caller's positions of the batch's boxes (after the tile tables)
const int *batch_pos(const Batch *bt) { return bt->d_off + (size_t)NFAM * (bt->ids.size() + 1); }

BatchDev bdev(const Batch *bt, int fam) {
  BatchDev d;
  d.boxes = bt->d_boxes;
  d.tile_off = bt->d_off + (size_t)fam * (bt->ids.size() + 1);
  d.nbox = (int)bt->ids.size();
  return d;
}

// The shared-memory attributes apply per device: set them once on each
// device the process uses (the current one).
int init_kernel_attrs() {
  static bool done[64] = {};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(AFID_EINVAL, "device %d out of range", dev);
  if (done[dev]) return 0;
  CK(cudaFuncSetAttribute(k_explicit_implicit_fwd<8, 2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, K1Ring<1, 8>::SMEM));
  CK(cudaFuncSetAttribute(k_explicit_implicit_fwd<8, 3, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, K1Ring<1, 8>::SMEM));
  CK(cudaFuncSetAttribute(k_explicit_implicit_fwd<8, 2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, K1Ring<2, 8>::SMEM));
  CK(cudaFuncSetAttribute(k_explicit_implicit_fwd<4, 4, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, K1Ring<1, 4>::SMEM));
  CK(cudaFuncSetAttribute(k_explicit_implicit_fwd<2, 8, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, K1Ring<1, 2>::SMEM));
  CK(cudaFuncSetAttribute(k_explicit_implicit_fwd<4, 5, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, K1Ring<1, 4>::SMEM));
  CK(cudaFuncSetAttribute(k_explicit_implicit_fwd<4, 6, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, K1Ring<1, 4>::SMEM));
  const int fsm = FFT_SMEM_MAX;   // two slots + work + twiddles: (4 N + 4) 16 bytes at one line
  CK(cudaFuncSetAttribute(k_fft_y_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fft_y_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fft_z<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fft_z<+1>, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fftw_y_fwd<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fftw_y_fwd<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fftw_y_inv<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fftw_y_inv<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fftw_z<-1, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fftw_z<-1, 12>, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fftw_z<+1, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  CK(cudaFuncSetAttribute(k_fftw_z<+1, 12>, cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  done[dev] = true;
  return 0;
}

// ---- launch sequences ------------------------------------------------------
// Optional per-kernel timing: when ``prof`` is set, an event is recorded
// after every launch and the elapsed times are accumulated per kernel slot.
struct Prof {
  std::vector<cudaEvent_t> ev;
  std::vector<int> slot;
  cudaStream_t s = nullptr;
  int mark(int k) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    CK(cudaEventRecord(e, s));
    ev.push_back(e);
    slot.push_back(k);
    return 0;
  }
};

#define PMARK(p, k)                 \
  do {                              \
    if (p) {                        \
      int r_ = (p)->mark(k);        \
      if (r_) return r_;            \
    }                               \
  } while (0)

// The x-solve of the Poisson equation (total[f] tiles of family f; bd(f)
// its descriptor).
template <class BD>
int launch_poisson_x(const int *total, BD bd, cudaStream_t s, int ns) {
  if (total[FAM_PX] > 0) {
    k_poisson_x<<<total[FAM_PX], 256, 0, s>>>(bd(FAM_PX), ns);
    CKL();
  }
  return 0;
}

int launch_poisson(const Batch *bt, cudaStream_t s, int ns, bool from_vel, Prof *pf = nullptr) {
  if (from_vel) {
    k_divergence<<<bt->total[FAM_COL], 256, 0, s>>>(bdev(bt, FAM_COL), ns);
    CKL();
    PMARK(pf, AFID_K_DIVERGENCE);
  }
  {
    int rc = launch_fft_y(true, bt->total, [&](int f) { return bdev(bt, f); }, bt->grid_y, bt->smem_y, bt->sm_y,
                          bt->grid_wy, bt->smem_wy, s, ns);
    if (rc) return rc;
  }
  PMARK(pf, AFID_K_FFT_Y_FWD);
  {
    int rc = launch_fft_z<-1>(bt->total, [&](int f) { return bdev(bt, f); }, bt->grid_z, bt->smem_z, bt->sm_z,
                              bt->grid_wz, bt->smem_wy, s, ns);
    if (rc) return rc;
  }
  PMARK(pf, AFID_K_FFT_Z_FWD);
  {
    int rc = launch_poisson_x(bt->total, [&](int fam) { return bdev(bt, fam); }, s, ns);
    if (rc) return rc;
  }
  PMARK(pf, AFID_K_POISSON_X);
  {
    int rc = launch_fft_z<+1>(bt->total, [&](int f) { return bdev(bt, f); }, bt->grid_z, bt->smem_z, bt->sm_z,
                              bt->grid_wz, bt->smem_wy, s, ns);
    if (rc) return rc;
  }
  PMARK(pf, AFID_K_FFT_Z_INV);
  {
    int rc = launch_fft_y(false, bt->total, [&](int f) { return bdev(bt, f); }, bt->grid_y, bt->smem_y, bt->sm_y,
                          bt->grid_wy, bt->smem_wy, s, ns);
    if (rc) return rc;
  }
  PMARK(pf, AFID_K_FFT_Y_INV);
  return 0;
}

int launch_substep(const Batch *bt, cudaStream_t s, int ns, Prof *pf = nullptr) {
  const int nb = (int)bt->ids.size();
  k_substep_prep<<<nb, 256, 0, s>>>(bt->d_boxes, nb, ns);
  CKL();
  PMARK(pf, AFID_K_PREP);
  const BatchDev k1 = bdev(bt, FAM_K1);
  const int nk1 = bt->total[FAM_K1];
  switch (bt->k1_minb) {
    case 3: k_explicit_implicit_fwd<8, 3, 1><<<nk1, 256, K1Ring<1, 8>::SMEM, s>>>(k1, ns); break;
    case 4: k_explicit_implicit_fwd<8, 2, 2><<<nk1, 256, K1Ring<2, 8>::SMEM, s>>>(k1, ns); break;
    case 5: k_explicit_implicit_fwd<4, 4, 1><<<nk1, 128, K1Ring<1, 4>::SMEM, s>>>(k1, ns); break;
    case 6: k_explicit_implicit_fwd<2, 8, 1><<<nk1, 64, K1Ring<1, 2>::SMEM, s>>>(k1, ns); break;
    case 7: k_explicit_implicit_fwd<4, 5, 1><<<nk1, 128, K1Ring<1, 4>::SMEM, s>>>(k1, ns); break;
    case 8: k_explicit_implicit_fwd<4, 6, 1><<<nk1, 128, K1Ring<1, 4>::SMEM, s>>>(k1, ns); break;
    default: k_explicit_implicit_fwd<8, 2, 1><<<nk1, 256, K1Ring<1, 8>::SMEM, s>>>(k1, ns); break;
  }
  CKL();
  PMARK(pf, AFID_K_EXPLICIT_FWD);
  k_implicit_bwd<<<bt->total[FAM_K2], bt->k2_block, 0, s>>>(bdev(bt, FAM_K2), ns);
  CKL();
  PMARK(pf, AFID_K_IMPLICIT_BWD);
  int rc = launch_poisson(bt, s, ns, true, pf);
  if (rc) return rc;
  k_correct<<<bt->total[FAM_COL], 256, 0, s>>>(bdev(bt, FAM_COL), ns, 1, 1);
  CKL();
  PMARK(pf, AFID_K_CORRECT);
  return 0;
}

int launch_step(const Batch *bt, cudaStream_t s, Prof *pf = nullptr) {
  const int nb = (int)bt->ids.size();
  k_diag<<<bt->total[FAM_DIAG], 256, 0, s>>>(bdev(bt, FAM_DIAG), 0);
  CKL();
  PMARK(pf, AFID_K_DIAG);
  k_finalize<<<cdiv(nb, 128), 128, 0, s>>>(bt->d_boxes, nb, 0);
  CKL();
  PMARK(pf, AFID_K_FINALIZE);
  for (int ns = 0; ns < 3; ++ns) {
    int rc = launch_substep(bt, s, ns, pf);
    if (rc) return rc;
  }
  k_plate_nu<<<dim3(NU_BLOCKS, nb), 256, 0, s>>>(bt->d_boxes, nb);
  CKL();
  PMARK(pf, AFID_K_PLATE_NU);
  k_finalize<<<cdiv(nb, 128), 128, 0, s>>>(bt->d_boxes, nb, 1);
  CKL();
  PMARK(pf, AFID_K_FINALIZE);
  return 0;
}

int field_ptr(HostBox *hb, int field, double **ptr, long long *rows, bool need_alloc) {
  BoxDev &d = hb->dev;
  *rows = d.nx;
  switch (field) {
    case AFID_VX: *ptr = d.vx; return 0;
    case AFID_VY: *ptr = d.vy; return 0;
    case AFID_VZ: *ptr = d.vz; return 0;
    case AFID_TEMP: *ptr = d.temp; return 0;
    case AFID_PR: *ptr = d.pr; return 0;
    case AFID_RUX: *ptr = d.rux; return 0;
    case AFID_RUY: *ptr = d.ruy; return 0;
    case AFID_RUZ: *ptr = d.ruz; return 0;
    case AFID_RUTEMP: *ptr = d.rutemp; return 0;
    case AFID_DPH: *ptr = d.phi; *rows = d.nxm; return 0;
    case AFID_WALL: *ptr = d.wall; *rows = 1; return 0;
    default: break;
  }
  if (field >= AFID_QCAP && field <= AFID_RHS) {
    if (!d.qcap) {
      if (!need_alloc) return fail(AFID_EINVAL, "routine buffers not allocated");
      return fail(AFID_EINVAL, "internal: routine buffers missing");
    }
    *ptr = field == AFID_QCAP ? d.qcap : field == AFID_DQ ? d.dq : field == AFID_HRO ? d.hro : d.rhs;
    return 0;
  }
  return fail(AFID_EINVAL, "unknown field %d", field);
}

int sync_self(HostBox *hb) {
  BoxDev d = hb->dev;
  d.active = 1;
  CK(cudaMemcpy(hb->d_self, &d, sizeof(BoxDev), cudaMemcpyHostToDevice));
  return 0;
}

int ensure_routine_bufs(afid_ctx *c, HostBox *hb) {
  if (hb->mem_routine) return 0;
  const size_t fs = (size_t)hb->dev.fsize;
  if (cudaMalloc(&hb->mem_routine, 4 * fs * sizeof(double)) != cudaSuccess)
    return fail(AFID_ENOMEM, "routine buffers: out of device memory");
  CK(cudaMemsetAsync(hb->mem_routine, 0, 4 * fs * sizeof(double), c->stream));
  double *r = (double *)hb->mem_routine;
  hb->dev.qcap = r; hb->dev.dq = r + fs; hb->dev.hro = r + 2 * fs; hb->dev.rhs = r + 3 * fs;
  // batches hold copies of the descriptor: drop them
  for (auto it = c->batches.begin(); it != c->batches.end();) {
    free_batch(it->second);
    it = c->batches.erase(it);
  }
  return sync_self(hb);
}

int single_batch(afid_ctx *c, int id, Batch **bt) { return get_batch(c, &id, 1, bt); }

}  // namespace

// ============================================================================
// C-ABI
// ============================================================================
extern "C" {

int afid_version(void) { return 10000; }

const char *afid_last_error(void) { return g_err.c_str(); }

int afid_ctx_create(afid_ctx **out, int device) {
  if (!out) return fail(AFID_EINVAL, "null ctx pointer");
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(AFID_EINVAL, "device %d out of range (%d)", device, ndev);
  afid_ctx *c = new afid_ctx();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail(AFID_ECUDA, "ctx create: %s", cudaGetErrorString(e));
  }
  c->stream = c->own;
  {
    const char *e = getenv("AFID_BATCH_STREAMS");
    if (e && atoi(e) == 1) c->split_sets = 0;
  }
  int rc = init_kernel_attrs();
  if (rc) { cudaStreamDestroy(c->own); delete c; return rc; }
  *out = c;
  return 0;
}

int afid_ctx_destroy(afid_ctx *c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (int h = 0; h < 2; ++h)
    if (c->side[h]) cudaStreamSynchronize(c->side[h]);
  for (auto &kv : c->batches) free_batch(kv.second);
  for (int h = 0; h < 2; ++h) {
    if (c->side[h]) cudaStreamDestroy(c->side[h]);
    if (c->ev_join[h]) cudaEventDestroy(c->ev_join[h]);
  }
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  for (auto &kv : c->rec_stage) {
    if (kv.second.d) cudaFree(kv.second.d);
    if (kv.second.h) cudaFreeHost(kv.second.h);
  }
  for (auto &kv : c->boxes) {
    HostBox *hb = kv.second;
    cudaFree(hb->mem_fields); cudaFree(hb->mem_scratch); cudaFree(hb->mem_small);
    cudaFree(hb->mem_routine); cudaFree(hb->d_self);
    delete hb;
  }
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return 0;
}

int afid_ctx_set_split_sets(afid_ctx *c, int on) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  c->split_sets = on ? 1 : 0;
  return 0;
}

int afid_ctx_set_stream(afid_ctx *c, void *stream) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  c->stream = stream ? (cudaStream_t)stream : c->own;
  return 0;
}

void *afid_ctx_stream(afid_ctx *c) { return c ? (void *)c->stream : nullptr; }

int afid_ctx_synchronize(afid_ctx *c) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int afid_make_grid(int nxm, int istr3, double str3, double alx3, double *xc) {
  if (nxm < 2 || !xc) return fail(AFID_EINVAL, "make_grid: nxm >= 2 and xc required");
  const int nx = nxm + 1;
  const double pi = 2.0 * std::asin(1.0);
  if (istr3 == 0) {
    for (int kc = 1; kc <= nx; ++kc) xc[kc - 1] = alx3 * ((double)(kc - 1) / (double)nxm);
  } else if (istr3 == 4) {
    const double tstr3 = std::tanh(str3);
    xc[0] = 0.0;
    for (int kc = 2; kc <= nx; ++kc) {
      const double z2dp = (double)(2 * kc - nx - 1) / (double)nxm;
      xc[kc - 1] = (1 + std::tanh(str3 * z2dp) / tstr3) * 0.5 * alx3;
      if (xc[kc - 1] < 0 || xc[kc - 1] > alx3) return fail(AFID_EINVAL, "grid is too stretched");
    }
  } else if (istr3 == 6) {
    const int nclip = (int)str3;
    const int nxmo = nx + nclip + nclip;
    std::vector<double> etaz(nx);
    for (int kc = 1; kc <= nx; ++kc)
      etaz[kc - 1] = std::cos(pi * ((double)(kc + nclip) - 0.5) / (double)nxmo);
    const double delet = etaz[0] - etaz[nx - 1];
    for (int kc = 1; kc <= nx; ++kc) etaz[kc - 1] = etaz[kc - 1] / (0.5 * delet);
    xc[0] = 0.0;
    for (int kc = 2; kc <= nxm; ++kc) xc[kc - 1] = alx3 * (1.0 - etaz[kc - 1]) * 0.5;
    xc[nx - 1] = alx3;
  } else if (istr3 == 7) {
    for (int kc = 1; kc <= nx; ++kc)
      xc[kc - 1] = alx3 * 0.5 * (1.0 - std::cos(pi * (double)(kc - 1) / (double)nxm));
    xc[0] = 0.0;
    xc[nx - 1] = alx3;
  } else {
    return fail(AFID_EINVAL, "istr3=%d not supported (0, 4, 6, 7)", istr3);
  }
  return 0;
}

size_t afid_box_device_bytes(const afid_box_params *p) {
  if (!p) return 0;
  Sizes s = sizes_of(*p);
  return (size_t)(9 * s.fsize + s.scratch + s.npiv + s.small) * sizeof(double) + 2 * sizeof(BoxDev) + 4096;
}

int afid_box_add(afid_ctx *c, const afid_box_params *p, const double *xc, int *box_id) {
  if (!c || !p || !xc || !box_id) return fail(AFID_EINVAL, "box_add: null argument");
  if (p->nxm < 3 || p->nym < 2 || p->nzm < 2) return fail(AFID_EINVAL, "box_add: nxm >= 3, nym, nzm >= 2");
  if (p->nym % 2) return fail(AFID_EINVAL, "box_add: nym must be even (real FFT along y)");
  if (p->nym > AFID_MAX_NYZ || p->nzm > AFID_MAX_NYZ)
    return fail(AFID_ESIZE, "box_add: nym, nzm <= %d (one transform line per block)", AFID_MAX_NYZ);
  if (p->nsst != 1 && p->nsst != 3) return fail(AFID_EINVAL, "box_add: nsst must be 1 or 3");
  if (!(p->ray > 0) || !(p->pra > 0) || !(p->ylen > 0) || !(p->zlen > 0) || !(p->alx3 > 0))
    return fail(AFID_EINVAL, "box_add: ray, pra, ylen, zlen, alx3 must be > 0");
  for (int k = 1; k <= p->nxm; ++k)
    if (!(xc[k] > xc[k - 1])) return fail(AFID_EINVAL, "box_add: xc must be increasing");
  int rc = set_device(c);
  if (rc) return rc;
  HostBox *hb = new HostBox();
  hb->prm = *p;
  BoxDev &d = hb->dev;
  d.nxm = p->nxm; d.nx = p->nxm + 1; d.nym = p->nym; d.nzm = p->nzm; d.nymh = p->nym / 2 + 1;
  d.nsst = p->nsst; d.inslws = p->inslws; d.inslwn = p->inslwn;
  if (factor_radices(d.nym, d.fft_y_radix, &d.fft_y_np) || factor_radices(d.nzm, d.fft_z_radix, &d.fft_z_np)) {
    delete hb;
    return fail(AFID_EFFT, "FFT size not efficient: nym=%d nzm=%d need prime factors <= 7 (code 444)", p->nym, p->nzm);
  }
  if (!warp_plan(d.nym, &d.wy_v, &d.wy_g, d.wy_rad, &d.wy_np, 2)) d.wy_v = 0;
  if (!warp_plan(d.nzm, &d.wz_v, &d.wz_g, d.wz_rad, &d.wz_np)) d.wz_v = 0;
  Sizes s = sizes_of(*p);
  d.plane = s.plane; d.fsize = s.fsize; d.nspec = s.nspec;
  d.dx = (double)p->nxm / p->alx3; d.dy = (double)p->nym / p->ylen; d.dz = (double)p->nzm / p->zlen;
  d.dxq = d.dx * d.dx; d.dyq = d.dy * d.dy; d.dzq = d.dz * d.dz;
  d.ren = std::sqrt(p->ray / p->pra);
  d.pec = std::sqrt(p->pra * p->ray);
  d.tempbp = p->tempbp; d.temptp = p->temptp;
  d.hist_cap = HIST_CAP;
  d.k1_minb = K1_DEFAULT;
  const size_t fb = 9 * (size_t)s.fsize * sizeof(double);
  const size_t sb = (size_t)(s.scratch + s.npiv) * sizeof(double);   // + the Poisson pivot table
  const size_t mb = (size_t)s.small * sizeof(double);
  if (cudaMalloc(&hb->mem_fields, fb) != cudaSuccess || cudaMalloc(&hb->mem_scratch, sb) != cudaSuccess ||
      cudaMalloc(&hb->mem_small, mb) != cudaSuccess || cudaMalloc(&hb->d_self, sizeof(BoxDev)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(hb->mem_fields); cudaFree(hb->mem_scratch); cudaFree(hb->mem_small); cudaFree(hb->d_self);
    delete hb;
    return fail(AFID_ENOMEM, "box_add: out of device memory (%zu bytes)", fb + sb + mb);
  }
  double *F = (double *)hb->mem_fields;
  d.vx = F; d.vy = F + s.fsize; d.vz = F + 2 * s.fsize; d.temp = F + 3 * s.fsize; d.pr = F + 4 * s.fsize;
  d.rux = F + 5 * s.fsize; d.ruy = F + 6 * s.fsize; d.ruz = F + 7 * s.fsize; d.rutemp = F + 8 * s.fsize;
  double *Sc = (double *)hb->mem_scratch;
  for (int q = 0; q < 4; ++q) d.ybuf[q] = Sc + q * s.fsize;
  d.spec = (double2 *)Sc;
  d.dstore = Sc + s.scratch;                 // pivot table, outside the aliased scratch
  d.phi = Sc + ((3 * s.nspec + 1) & ~1LL);   // 16-byte aligned rows for the bulk copies
  hb->scratch_doubles = (size_t)s.scratch;
  // small allocations
  double *M = (double *)hb->mem_small;
  size_t o = 0;
  std::vector<double> tab;
  build_tables(*p, xc, tab);
  d.tab = M + o; o += tab.size();
  o = (o + 1) & ~(size_t)1;
  d.twy = (const double2 *)(M + o); o += 2 * (size_t)p->nym;
  d.twz = (const double2 *)(M + o); o += 2 * (size_t)p->nzm;
  d.coef = M + o; o += (size_t)SYS_N * C_N * d.nx;
  d.nu_part = M + o; o += 2 * NU_BLOCKS;
  d.hist = M + o; o += (size_t)HIST_CAP * HIST_FIELDS;
  d.wall = M + o; o += (size_t)s.plane;
  o = (o + 7) & ~(size_t)7;
  d.sc = (BoxScalars *)(M + o); o += (sizeof(BoxScalars) + 63) / 8;
  o = (o + 7) & ~(size_t)7;   // 64-byte aligned (mem_small is 256-byte aligned)
  d.tm_z = (const CUtensorMap *)(M + o); o += sizeof(CUtensorMap) / 8;
  if ((long long)o > s.small) {
    cudaFree(hb->mem_fields); cudaFree(hb->mem_scratch); cudaFree(hb->mem_small); cudaFree(hb->d_self);
    delete hb;
    return fail(AFID_ECUDA, "box_add: small-region layout exceeds its allocation");
  }
  std::vector<double2> tw((size_t)p->nym + p->nzm);
  build_twiddles(p->nym, tw.data());
  build_twiddles(p->nzm, tw.data() + p->nym);
  BoxScalars bs;
  memset(&bs, 0, sizeof bs);
  bs.dt = p->dt; bs.idtv = p->idtv; bs.cflmax = p->cflmax; bs.dtmin = p->dtmin; bs.dtmax = p->dtmax;
  bs.limitvel = p->vlim; bs.resid = p->resid;
  cudaStream_t st = c->stream;
  bool ok = cudaMemsetAsync(hb->mem_fields, 0, fb, st) == cudaSuccess &&
            cudaMemsetAsync(hb->mem_scratch, 0, sb, st) == cudaSuccess &&
            cudaMemsetAsync(hb->mem_small, 0, mb, st) == cudaSuccess &&
            cudaMemcpyAsync((void *)d.tab, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync((void *)d.twy, tw.data(), tw.size() * 16, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(d.sc, &bs, sizeof bs, cudaMemcpyHostToDevice, st) == cudaSuccess;
  if (ok) {   // the Poisson pivots depend on the grid only: tabulate them once
    k_poisson_pivots<<<(unsigned)cdiv(px_pairs(p->nzm, d.nymh), 256), 256, 0, st>>>(d);
    ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess;
    d.piv_ready = 1;
  }
  if (!ok) {
    cudaFree(hb->mem_fields); cudaFree(hb->mem_scratch); cudaFree(hb->mem_small); cudaFree(hb->d_self);
    delete hb;
    return fail(AFID_ECUDA, "box_add: initialisation copy failed");
  }
  rc = write_z_map(hb->dev, st);
  if (rc) {
    cudaFree(hb->mem_fields); cudaFree(hb->mem_scratch); cudaFree(hb->mem_small); cudaFree(hb->d_self);
    delete hb;
    return rc;
  }
  hb->id = c->next_id++;
  hb->xc.assign(xc, xc + p->nxm + 1);
  hb->stats.assign((size_t)AFID_NSTAT * p->nxm, 0.0);
  rc = sync_self(hb);
  if (rc) return rc;
  c->boxes[hb->id] = hb;
  *box_id = hb->id;
  return 0;
}

int afid_box_remove(afid_ctx *c, int id) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto it = c->batches.begin(); it != c->batches.end();) {
    bool has = false;
    for (int x : it->first) has |= (x == id);
    if (has) { free_batch(it->second); it = c->batches.erase(it); }
    else ++it;
  }
  cudaFree(hb->mem_fields); cudaFree(hb->mem_scratch); cudaFree(hb->mem_small);
  cudaFree(hb->mem_routine); cudaFree(hb->d_self); cudaFree(hb->d_out);
  c->boxes.erase(id);
  delete hb;
  return 0;
}

static int transfer(afid_ctx *c, int id, int field, double *host, bool up, bool sync = true) {
  if (!c || !host) return fail(AFID_EINVAL, "null argument");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  if (field >= AFID_QCAP && field <= AFID_RHS) {
    rc = ensure_routine_bufs(c, hb);
    if (rc) return rc;
  }
  double *dp;
  long long rows;
  rc = field_ptr(hb, field, &dp, &rows, true);
  if (rc) return rc;
  const BoxDev &d = hb->dev;
  cudaStream_t st = c->stream;
  if (field == AFID_WALL) {
    const size_t bytes = (size_t)d.plane * sizeof(double);
    if (up) CK(cudaMemcpyAsync(dp, host, bytes, cudaMemcpyHostToDevice, st));
    else CK(cudaMemcpyAsync(host, dp, bytes, cudaMemcpyDeviceToHost, st));
    if (sync) CK(cudaStreamSynchronize(st));
    return 0;
  }
  const size_t n = (size_t)rows * d.plane;
  // staging: the first scratch field (the forward-sweep buffer of vx), which
  // never overlaps dph
  double *stg = d.ybuf[0];
  if (field == AFID_DPH) stg = d.ybuf[0];
  dim3 blk(32, 8);
  dim3 grd((unsigned)cdiv(rows, 32), (unsigned)cdiv(d.nym, 32), (unsigned)d.nzm);
  if (up) {
    CK(cudaMemcpyAsync(stg, host, n * sizeof(double), cudaMemcpyHostToDevice, st));
    k_fortran_to_dev<<<grd, blk, 0, st>>>(stg, dp, (int)rows, d.nym, d.nzm, (int)rows);
    CKL();
  } else {
    k_dev_to_fortran<<<grd, blk, 0, st>>>(dp, stg, (int)rows, d.nym, d.nzm, (int)rows);
    CKL();
    CK(cudaMemcpyAsync(host, stg, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  if (sync) CK(cudaStreamSynchronize(st));
  return 0;
}

int afid_box_upload(afid_ctx *c, int id, int field, const double *host) {
  return transfer(c, id, field, const_cast<double *>(host), true);
}

int afid_box_download(afid_ctx *c, int id, int field, double *host) {
  return transfer(c, id, field, host, false);
}

// The same copies queued on the context's stream without waiting: the
// box's staging buffer is reused by the next transfer of the same box in
// stream order, so queued transfers of one box do not overwrite each other.
int afid_box_upload_async(afid_ctx *c, int id, int field, const double *host) {
  return transfer(c, id, field, const_cast<double *>(host), true, false);
}

int afid_box_download_async(afid_ctx *c, int id, int field, double *host) {
  return transfer(c, id, field, host, false, false);
}

__global__ void k_reset_box(double *hist, long long nh, double *wall, long long nw, BoxScalars *S, double dt) {
  const long long n = nh + nw;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    if (e < nh) hist[e] = 0.0;
    else wall[e - nh] = 0.0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S->time = 0.0;
    S->ntime = 0;
    S->status = 0;
    S->nonfinite = 0;
    for (int q = 0; q < 4; ++q) S->red_u64[q] = 0ull;
    if (dt > 0) S->dt = dt;
  }
}

int afid_box_reset(afid_ctx *c, int id, double dt) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  const BoxDev &d = hb->dev;
  cudaStream_t st = c->stream;
  // the RK history and wall row zeroed and the record reset by one kernel
  // in stream order: no host round trip, and no memset, which may queue on a
  // copy engine behind other streams' transfers
  const long long nh = 4 * d.fsize, nw = d.plane;
  k_reset_box<<<(unsigned)std::min<long long>(cdiv(nh + nw, 256), 4096), 256, 0, st>>>(d.rux, nh, d.wall, nw,
                                                                                       d.sc, dt);
  CKL();
  return 0;
}

int afid_box_set_time(afid_ctx *c, int id, double time) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  CK(cudaMemcpyAsync((char *)hb->dev.sc + offsetof(BoxScalars, time), &time, sizeof time,
                     cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// ---- restart onto a new grid (ReadFlowField.F90:63-150, interp.F90) ------
// gridnew (interp.F90:229-296): nodes rc and centres rm of an n-point grid on
// [0, rext] for istr 0 and 6 (for those, CreateGrid's nodes), indexed 0..n+1
// with the second-order extrapolated ends of interp.F90:45-60
static int gridnew_pad(int n, double rext, int istr, double stri, std::vector<double> &rc, std::vector<double> &rm) {
  rc.assign(n + 2, 0.0);
  rm.assign(n + 2, 0.0);
  if (afid_make_grid(n - 1, istr, stri, rext, rc.data() + 1)) return -1;
  for (int i = 1; i < n; ++i) rm[i] = (rc[i] + rc[i + 1]) * 0.5;
  rm[n] = 2 * rc[n] - rm[n - 1];
  for (std::vector<double> *v : {&rc, &rm}) {
    std::vector<double> &a = *v;
    a[0] = 2 * a[1] - a[2];
    a[n + 1] = 2 * a[n] - a[n - 1];
  }
  return 0;
}

// per new coordinate: the new value, the bracketing old values and indices
// (interp.F90:128-175), as five rows of length m at t
static void interp_axis(const std::vector<double> &oldc, int n, const std::vector<double> &newc, int m, double *t) {
  for (int q = 0; q < m; ++q) {
    const double b = newc[q + 1];
    int f = n - 1, cc = n;
    for (int l = 1; l <= n; ++l)
      if (oldc[l] >= b) { f = l - 1; cc = l; break; }
    t[q] = b; t[m + q] = oldc[f]; t[2 * m + q] = oldc[cc]; t[3 * m + q] = f; t[4 * m + q] = cc;
  }
}

int afid_box_interp_field(afid_ctx *c, int id, int field, const double *old, int nxo, int nyo, int nzo,
                          int istro3, double stro3, int istr3, double str3) {
  if (!c || !old) return fail(AFID_EINVAL, "interp_field: null argument");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  // interp.F90's case per field as ReadFlowField.F90:70-73 numbers them
  // (vxflag = 1 ... teflag = 4); case 1 is staggered in z and case 3 in x
  int flag;
  switch (field) {
    case AFID_VX: flag = 1; break;
    case AFID_VY: flag = 2; break;
    case AFID_VZ: flag = 3; break;
    case AFID_TEMP: flag = 4; break;
    default: return fail(AFID_EINVAL, "interp_field: field must be vx, vy, vz or temp");
  }
  const afid_box_params &p = hb->prm;
  const int nx = p.nxm + 1, ny = p.nym + 1, nz = p.nzm + 1;
  if (nz > nzo * 2 || ny > nyo * 2 || nx > nxo * 2)   // ReadFlowField.F90:88-99
    return fail(AFID_EINVAL, "interp_field: new grid resolution cannot be more than twice the old resolution");
  if (nxo < 3 || nyo < 3 || nzo < 3) return fail(AFID_EINVAL, "interp_field: old grid too small (nx, ny, nz >= 3)");
  if ((istro3 != 0 && istro3 != 6) || (istr3 != 0 && istr3 != 6))
    return fail(AFID_EINVAL, "interp_field: interp.F90's gridnew defines istr3 0 and 6 only (got %d, %d)", istro3, istr3);
  std::vector<double> tco, tmo, rco, rmo, zzo, zmo, tcn, tmn, rcn, rmn, zzn, zmn;
  if (gridnew_pad(nzo, p.zlen, 0, 1.0, tco, tmo) || gridnew_pad(nyo, p.ylen, 0, 1.0, rco, rmo) ||
      gridnew_pad(nxo, 1.0, istro3, stro3, zzo, zmo) || gridnew_pad(nz, p.zlen, 0, 1.0, tcn, tmn) ||
      gridnew_pad(ny, p.ylen, 0, 1.0, rcn, rmn) || gridnew_pad(nx, 1.0, istr3, str3, zzn, zmn))
    return fail(AFID_EINVAL, "interp_field: grid construction failed");
  const std::vector<double> &xo = flag == 1 ? tco : tmo, &xn = flag == 1 ? tcn : tmn;
  const std::vector<double> &yo = flag == 2 ? rco : rmo, &yn = flag == 2 ? rcn : rmn;
  const std::vector<double> &zo = flag == 3 ? zzo : zmo, &zn = flag == 3 ? zzn : zmn;
  const int nzm = p.nzm, nym = p.nym, nyom = nyo - 1, nzom = nzo - 1;
  const size_t ntab = 5 * ((size_t)nzm + nym + nx), nold = (size_t)nxo * nyom * nzom;
  std::vector<double> tab(ntab);
  interp_axis(xo, nzo, xn, nzm, tab.data());
  interp_axis(yo, nyo, yn, nym, tab.data() + 5 * (size_t)nzm);
  interp_axis(zo, nxo, zn, nx, tab.data() + 5 * ((size_t)nzm + nym));
  rc = set_device(c);
  if (rc) return rc;
  double *buf = nullptr;
  if (cudaMalloc(&buf, (ntab + nold) * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return fail(AFID_ENOMEM, "interp_field: %zu bytes of device memory", (ntab + nold) * sizeof(double));
  }
  const BoxDev &d = hb->dev;
  double *dst = field == AFID_VX ? d.vx : field == AFID_VY ? d.vy : field == AFID_VZ ? d.vz : d.temp;
  const long long npt = (long long)nx * nym * nzm;
  cudaStream_t st = c->stream;
  bool ok = cudaMemcpyAsync(buf, tab.data(), ntab * sizeof(double), cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(buf + ntab, old, nold * sizeof(double), cudaMemcpyHostToDevice, st) == cudaSuccess;
  if (ok) {
    k_interp<<<(unsigned)((npt + 255) / 256), 256, 0, st>>>(buf + ntab, nxo, nyom, nzom, buf, dst, nx, nym, nzm);
    ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess;
  }
  cudaFree(buf);
  if (!ok) return fail(AFID_ECUDA, "interp_field: copy or kernel failed");
  return 0;
}

// The record staging of the context's current stream, grown to n records
// (growing waits for the stream first: a queued copy may still read it).
// The pinned host half is made only when a caller needs it (the waiting
// read): allocating pinned memory can stall the whole device, which the
// queued read must not do after its first call on a stream.
static int rec_stage(afid_ctx *c, int n, bool host, afid_ctx::RecStage **out) {
  afid_ctx::RecStage &rs = c->rec_stage[c->stream];
  if (n > rs.n || (host && !rs.h)) {
    CK(cudaStreamSynchronize(c->stream));
    const int m = n > rs.n ? n : rs.n;
    if (rs.d) cudaFree(rs.d);
    if (rs.h) cudaFreeHost(rs.h);
    rs.d = nullptr;
    rs.h = nullptr;
    rs.n = 0;
    if (cudaMalloc(&rs.d, sizeof(BoxScalars) * m) != cudaSuccess ||
        (host && cudaMallocHost(&rs.h, sizeof(BoxScalars) * m) != cudaSuccess))
      return fail(AFID_ENOMEM, "record staging of %d records", m);
    rs.n = m;
  }
  *out = &rs;
  return 0;
}

static void scalars_out(const BoxScalars &bs, afid_box_scalars *out) {
  out->dt = bs.dt; out->time = bs.time; out->cfl = bs.cfl; out->cfl_used = bs.cfl_used;
  out->divmax = bs.divmax;
  for (int q = 0; q < 3; ++q) out->vmax[q] = bs.vmax[q];
  out->nu_bot = bs.nu_bot; out->nu_top = bs.nu_top; out->ntime = bs.ntime; out->status = bs.status;
}

__global__ void k_gather_scalars(const BoxDev *boxes, const int *pos, int n, BoxScalars *dst) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n) dst[pos[b]] = *boxes[b].sc;
}

// the public records of n boxes, written straight in afid_box_scalars layout
__global__ void k_gather_records(const BoxDev *boxes, const int *pos, int n, afid_box_scalars *dst) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const BoxScalars &bs = *boxes[b].sc;
  afid_box_scalars o;
  o.dt = bs.dt; o.time = bs.time; o.cfl = bs.cfl; o.cfl_used = bs.cfl_used; o.divmax = bs.divmax;
  for (int q = 0; q < 3; ++q) o.vmax[q] = bs.vmax[q];
  o.nu_bot = bs.nu_bot; o.nu_top = bs.nu_top; o.ntime = bs.ntime; o.status = bs.status;
  dst[pos[b]] = o;
}

int afid_boxes_get_scalars(afid_ctx *c, const int *ids, int n, afid_box_scalars *out) {
  if (!c || !ids || !out || n <= 0) return fail(AFID_EINVAL, "boxes_get_scalars: null argument or n <= 0");
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = get_batch(c, ids, n, &bt);
  if (rc) return rc;
  afid_ctx::RecStage *rs;
  rc = rec_stage(c, n, true, &rs);
  if (rc) return rc;
  k_gather_scalars<<<(unsigned)cdiv(n, 128), 128, 0, c->stream>>>(bt->d_boxes, batch_pos(bt), n, rs->d);
  CKL();
  CK(cudaMemcpyAsync(rs->h, rs->d, sizeof(BoxScalars) * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int b = 0; b < n; ++b) scalars_out(rs->h[b], out + b);
  return 0;
}

int afid_boxes_get_scalars_async(afid_ctx *c, const int *ids, int n, afid_box_scalars *out) {
  if (!c || !ids || !out || n <= 0) return fail(AFID_EINVAL, "boxes_get_scalars_async: null argument or n <= 0");
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = get_batch(c, ids, n, &bt);
  if (rc) return rc;
  // the stream's staging array serves every call on it: each call's copy is
  // queued right behind its gather, and the next call's gather behind that
  // copy, so no record is overwritten before it is copied
  // pinned host memory the device can reach: the gather writes the records
  // there itself, so the read puts no copy on a copy engine (where it could
  // wait behind other streams' transfers)
  {
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, out) == cudaSuccess && pa.type == cudaMemoryTypeHost && pa.devicePointer) {
      k_gather_records<<<(unsigned)cdiv(n, 128), 128, 0, c->stream>>>(bt->d_boxes, batch_pos(bt), n,
                                                                     (afid_box_scalars *)pa.devicePointer);
      CKL();
      return 0;
    }
    cudaGetLastError();   // pageable memory: not an error
  }
  const size_t need = (sizeof(afid_box_scalars) * n + sizeof(BoxScalars) - 1) / sizeof(BoxScalars);
  afid_ctx::RecStage *rs;
  rc = rec_stage(c, (int)need, false, &rs);
  if (rc) return rc;
  afid_box_scalars *d = reinterpret_cast<afid_box_scalars *>(rs->d);
  k_gather_records<<<(unsigned)cdiv(n, 128), 128, 0, c->stream>>>(bt->d_boxes, batch_pos(bt), n, d);
  CKL();
  CK(cudaMemcpyAsync(out, d, sizeof(afid_box_scalars) * n, cudaMemcpyDeviceToHost, c->stream));
  return 0;
}

int afid_box_get_scalars(afid_ctx *c, int id, afid_box_scalars *out) {
  if (!c || !out) return fail(AFID_EINVAL, "null argument");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  BoxScalars bs;
  CK(cudaMemcpyAsync(&bs, hb->dev.sc, sizeof bs, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  scalars_out(bs, out);
  return 0;
}

int afid_box_set_stop(afid_ctx *c, int id, int stop_ntime, double tout, double tmax) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  static_assert(AFID_STATUS_HELD == AFID_STATUS_HELD_DEV, "hold status of the C-ABI and the kernels");
  const int stop = stop_ntime > 0 ? stop_ntime : 0;
  const double to = tout > 0 ? tout : 0.0, tm = tmax > 0 ? tmax : 0.0;
  char *sc = (char *)hb->dev.sc;
  CK(cudaMemcpyAsync(sc + offsetof(BoxScalars, stop_ntime), &stop, sizeof stop, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(sc + offsetof(BoxScalars, tout), &to, sizeof to, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(sc + offsetof(BoxScalars, tmax), &tm, sizeof tm, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int afid_box_test_skip_z_copies(afid_ctx *c, int id, int skip, unsigned max_polls) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  hb->dev.z_copy_skip = skip ? 1 : 0;
  hb->dev.mbar_tries = max_polls;
  // the switch acts on the tile z kernel: a skipped box leaves the warp plan
  BoxDev &d = hb->dev;
  if (skip || !warp_plan(d.nzm, &d.wz_v, &d.wz_g, d.wz_rad, &d.wz_np)) d.wz_v = 0;
  // batches hold copies of the descriptor: drop the ones with this box
  for (auto it = c->batches.begin(); it != c->batches.end();) {
    bool has = false;
    for (int x : it->first) has |= (x == id);
    if (has) { free_batch(it->second); it = c->batches.erase(it); }
    else ++it;
  }
  return sync_self(hb);
}

int afid_box_resume(afid_ctx *c, int id) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  k_resume<<<1, 32, 0, c->stream>>>(hb->d_self, 1);
  CKL();
  return 0;
}

int afid_box_history(afid_ctx *c, int id, afid_step_record *out, int max_records) {
  if (!c || !out || max_records < 0) return fail(AFID_EINVAL, "bad argument");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  BoxScalars bs;
  CK(cudaMemcpyAsync(&bs, hb->dev.sc, sizeof bs, cudaMemcpyDeviceToHost, c->stream));
  std::vector<double> h((size_t)HIST_CAP * HIST_FIELDS);
  CK(cudaMemcpyAsync(h.data(), hb->dev.hist, h.size() * 8, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int avail = bs.ntime < HIST_CAP ? bs.ntime : HIST_CAP;
  int n = avail < max_records ? avail : max_records;
  for (int r = 0; r < n; ++r) {
    const int step = bs.ntime - n + r;               // 0-based step index
    const double *src = &h[(size_t)(step % HIST_CAP) * HIST_FIELDS];
    out[r].time = src[0]; out[r].dt = src[1]; out[r].cfl_used = src[2]; out[r].divmax = src[3];
    out[r].nu_bot = src[4]; out[r].nu_top = src[5]; out[r].vmax_y = src[6]; out[r].vmax_z = src[7];
  }
  return n;
}

int afid_box_set_tuning(afid_ctx *c, int id, int fft_y_lines, int fft_z_lines, int k1_minb) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  BoxDev &d = hb->dev;
  if (fft_y_lines < 0 || (fft_y_lines > 0 && !fft_y_ok(d.nym, fft_y_lines, FFT_SMEM_MAX)))
    return fail(AFID_EINVAL, "fft_y_lines %d out of range", fft_y_lines);
  if (fft_z_lines < 0 || (fft_z_lines > 0 && !fft_z_ok(d.nzm, fft_z_lines, FFT_SMEM_MAX)))
    return fail(AFID_EINVAL, "fft_z_lines %d out of range", fft_z_lines);
  if (k1_minb != 0 && (k1_minb < K1_VMIN || k1_minb > K1_VMAX))
    return fail(AFID_EINVAL, "k1 variant must be 0 or %d..%d", K1_VMIN, K1_VMAX);
  rc = set_device(c);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  d.fy_lines = fft_y_lines;
  d.fz_lines = fft_z_lines;
  d.k1_minb = k1_minb ? k1_minb : K1_DEFAULT;
  rc = write_z_map(d, c->stream);   // the TMA box width follows the z lines
  if (rc) return rc;
  // batches hold copies of the descriptor and tile tables: drop them
  for (auto it = c->batches.begin(); it != c->batches.end();) {
    bool has = false;
    for (int x : it->first) has |= (x == id);
    if (has) { free_batch(it->second); it = c->batches.erase(it); }
    else ++it;
  }
  return sync_self(hb);
}

// ---- routine-level entry points -------------------------------------------
int afid_time_marcher_begin_substep(afid_ctx *c, int id, int ns) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  if (ns < 0 || ns >= hb->prm.nsst) return fail(AFID_EINVAL, "substep %d out of range", ns);
  rc = set_device(c);
  if (rc) return rc;
  k_substep_prep<<<1, 256, 0, c->stream>>>(hb->d_self, 1, ns);
  CKL();
  return 0;
}

static int explicit_one(afid_ctx *c, int id, int field) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  rc = ensure_routine_bufs(c, hb);
  if (rc) return rc;
  const BoxDev &d = hb->dev;
  k_explicit_one<<<(unsigned)cdiv((long long)d.nxm * d.plane, 256), 256, 0, c->stream>>>(hb->d_self, field);
  CKL();
  return 0;
}

static int implicit_one(afid_ctx *c, int id, int field) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  rc = ensure_routine_bufs(c, hb);
  if (rc) return rc;
  const BoxDev &d = hb->dev;
  k_implicit_one<<<(unsigned)cdiv(d.plane, 256), 256, 0, c->stream>>>(hb->d_self, field);
  CKL();
  return 0;
}

int afid_explicit_terms_vx(afid_ctx *c, int id) { return explicit_one(c, id, F_VX); }
int afid_explicit_terms_vy(afid_ctx *c, int id) { return explicit_one(c, id, F_VY); }
int afid_explicit_terms_vz(afid_ctx *c, int id) { return explicit_one(c, id, F_VZ); }
int afid_explicit_terms_temp(afid_ctx *c, int id) { return explicit_one(c, id, F_T); }
int afid_implicit_and_update_vx(afid_ctx *c, int id) { return implicit_one(c, id, F_VX); }
int afid_implicit_and_update_vy(afid_ctx *c, int id) { return implicit_one(c, id, F_VY); }
int afid_implicit_and_update_vz(afid_ctx *c, int id) { return implicit_one(c, id, F_VZ); }
int afid_implicit_and_update_temp(afid_ctx *c, int id) { return implicit_one(c, id, F_T); }

int afid_calc_local_divergence(afid_ctx *c, int id) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = single_batch(c, id, &bt);
  if (rc) return rc;
  k_divergence<<<bt->total[FAM_COL], 256, 0, c->stream>>>(bdev(bt, FAM_COL), 0);
  CKL();
  return 0;
}

int afid_solve_pressure_correction(afid_ctx *c, int id) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = single_batch(c, id, &bt);
  if (rc) return rc;
  return launch_poisson(bt, c->stream, 0, false);
}

static int correct(afid_ctx *c, int id, int vel, int pr) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = single_batch(c, id, &bt);
  if (rc) return rc;
  k_correct<<<bt->total[FAM_COL], 256, 0, c->stream>>>(bdev(bt, FAM_COL), 0, vel, pr);
  CKL();
  return 0;
}

int afid_correct_velocity(afid_ctx *c, int id) { return correct(c, id, 1, 0); }
int afid_correct_pressure(afid_ctx *c, int id) { return correct(c, id, 0, 1); }

static int diag_now(afid_ctx *c, int id, BoxScalars *bs) {
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = single_batch(c, id, &bt);
  if (rc) return rc;
  HostBox *hb;
  rc = get_box(c, id, &hb);
  if (rc) return rc;
  void *red = (char *)hb->dev.sc + offsetof(BoxScalars, red_u64);
  CK(cudaMemsetAsync(red, 0, sizeof(bs->red_u64), c->stream));
  k_diag<<<bt->total[FAM_DIAG], 256, 0, c->stream>>>(bdev(bt, FAM_DIAG), 1);
  CKL();
  CK(cudaMemcpyAsync(bs, hb->dev.sc, sizeof(BoxScalars), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemsetAsync(red, 0, sizeof(bs->red_u64), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int afid_calc_max_cfl(afid_ctx *c, int id, double *cflm) {
  if (!c || !cflm) return fail(AFID_EINVAL, "null argument");
  BoxScalars bs;
  int rc = diag_now(c, id, &bs);
  if (rc) return rc;
  double v;
  long long bits = (long long)bs.red_u64[0];
  memcpy(&v, &bits, 8);
  *cflm = v > 0.00000001 ? v : 0.00000001;
  return 0;
}

int afid_check_divergence(afid_ctx *c, int id, double *qmax) {
  if (!c || !qmax) return fail(AFID_EINVAL, "null argument");
  BoxScalars bs;
  int rc = diag_now(c, id, &bs);
  if (rc) return rc;
  long long bits = (long long)bs.red_u64[1];
  memcpy(qmax, &bits, 8);
  return 0;
}

int afid_calc_plate_nu(afid_ctx *c, int id, double *nuslow, double *nusupp) {
  if (!c || !nuslow || !nusupp) return fail(AFID_EINVAL, "null argument");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  rc = set_device(c);
  if (rc) return rc;
  k_plate_nu<<<dim3(NU_BLOCKS, 1), 256, 0, c->stream>>>(hb->d_self, 1);
  CKL();
  double part[2 * NU_BLOCKS];
  CK(cudaMemcpyAsync(part, hb->dev.nu_part, sizeof part, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double lo = 0.0, up = 0.0;
  for (int q = 0; q < NU_BLOCKS; ++q) { lo += part[2 * q]; up += part[2 * q + 1]; }
  *nuslow = lo / (double)(hb->dev.nzm * hb->dev.nym);
  *nusupp = up / (double)(hb->dev.nzm * hb->dev.nym);
  return 0;
}

// ---- fused path ---------------------------------------------------------------
int afid_substep(afid_ctx *c, const int *ids, int n, int ns) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  if (ns < 0 || ns > 2) return fail(AFID_EINVAL, "substep %d out of range", ns);
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = get_batch(c, ids, n, &bt);
  if (rc) return rc;
  return launch_substep(bt, c->stream, ns);
}

int afid_step(afid_ctx *c, const int *ids, int n, int nsteps) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  if (nsteps < 0) return fail(AFID_EINVAL, "nsteps < 0");
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = get_batch(c, ids, n, &bt);
  if (rc) return rc;
  for (int s = 0; s < nsteps; ++s) {
    rc = launch_step(bt, c->stream);
    if (rc) return rc;
  }
  return 0;
}

int afid_step_profiled(afid_ctx *c, const int *ids, int n, int nsteps, double *kernel_ms,
                       int *kernel_launches, int nkernel) {
  if (!c || !kernel_ms || nkernel < AFID_K_COUNT) return fail(AFID_EINVAL, "bad argument");
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = get_batch(c, ids, n, &bt);
  if (rc) return rc;
  for (int k = 0; k < nkernel; ++k) { kernel_ms[k] = 0.0; if (kernel_launches) kernel_launches[k] = 0; }
  for (int st = 0; st < nsteps; ++st) {
    Prof pf;
    pf.s = c->stream;
    rc = pf.mark(-1);
    if (rc) return rc;
    rc = launch_step(bt, c->stream, &pf);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    for (size_t q = 1; q < pf.ev.size(); ++q) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, pf.ev[q - 1], pf.ev[q]));
      kernel_ms[pf.slot[q]] += ms;
      if (kernel_launches) kernel_launches[pf.slot[q]] += 1;
    }
    for (auto e : pf.ev) cudaEventDestroy(e);
  }
  return 0;
}

}  // extern "C"

namespace {

// The step graph of batch bt for stream st (captured on first use, and
// again when the stream changes).
int ensure_graph(Batch *bt, cudaStream_t st) {
  if (bt->gexec && bt->gstream == st) return 0;
  if (bt->gexec) { cudaGraphExecDestroy(bt->gexec); bt->gexec = nullptr; }
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  int rc = launch_step(bt, st);
  cudaError_t e = cudaStreamEndCapture(st, &g);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(AFID_ECUDA, "graph capture: %s", cudaGetErrorString(e));
  size_t nn = 0;
  e = cudaGraphGetNodes(g, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn);
  if (e == cudaSuccess && nn) e = cudaGraphGetNodes(g, nodes.data(), &nn);
  int nk = 0;
  for (size_t q = 0; e == cudaSuccess && q < nn; ++q) {
    cudaGraphNodeType t;
    e = cudaGraphNodeGetType(nodes[q], &t);
    if (e == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nk;
  }
  if (e != cudaSuccess) { cudaGraphDestroy(g); return fail(AFID_ECUDA, "graph nodes: %s", cudaGetErrorString(e)); }
  e = cudaGraphInstantiate(&bt->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { bt->gexec = nullptr; return fail(AFID_ECUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
  bt->gstream = st;
  bt->graph_kernels = nk;
  return 0;
}

// The streams and events of split batches.
int ensure_side(afid_ctx *c) {
  for (int h = 0; h < 2; ++h)
    if (!c->side[h]) CK(cudaStreamCreateWithFlags(&c->side[h], cudaStreamNonBlocking));
  if (!c->ev_fork) CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  for (int h = 0; h < 2; ++h)
    if (!c->ev_join[h]) CK(cudaEventCreateWithFlags(&c->ev_join[h], cudaEventDisableTiming));
  return 0;
}

// The halves of a split batch with their graphs on the side streams.
int split_halves(afid_ctx *c, const Batch *bt, Batch **hb) {
  int rc = ensure_side(c);
  for (int h = 0; !rc && h < 2; ++h) {
    rc = get_batch(c, bt->half_ids[h].data(), (int)bt->half_ids[h].size(), &hb[h], false);
    if (!rc) rc = ensure_graph(hb[h], c->side[h]);
  }
  return rc;
}

}  // namespace

extern "C" {

int afid_step_graph(afid_ctx *c, const int *ids, int n, int nsteps) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  if (nsteps < 0) return fail(AFID_EINVAL, "nsteps < 0");
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = get_batch(c, ids, n, &bt);
  if (rc) return rc;
  if (bt->split && c->split_sets) {
    // each half steps on its own stream between a fork from and a join to
    // the context's stream; the halves are independent, so they need no
    // other ordering
    Batch *hb[2];
    rc = split_halves(c, bt, hb);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev_fork, c->stream));
    for (int h = 0; h < 2; ++h) CK(cudaStreamWaitEvent(c->side[h], c->ev_fork, 0));
    for (int s = 0; s < nsteps; ++s)
      for (int h = 0; h < 2; ++h) CK(cudaGraphLaunch(hb[h]->gexec, c->side[h]));
    for (int h = 0; h < 2; ++h) {
      CK(cudaEventRecord(c->ev_join[h], c->side[h]));
      CK(cudaStreamWaitEvent(c->stream, c->ev_join[h], 0));
    }
    return 0;
  }
  rc = ensure_graph(bt, c->stream);
  if (rc) return rc;
  for (int s = 0; s < nsteps; ++s) CK(cudaGraphLaunch(bt->gexec, c->stream));
  return 0;
}

int afid_step_graph_kernels(afid_ctx *c, const int *ids, int n, int *kernels) {
  if (!c || !kernels) return fail(AFID_EINVAL, "null argument");
  int rc = set_device(c);
  if (rc) return rc;
  Batch *bt;
  rc = get_batch(c, ids, n, &bt);
  if (rc) return rc;
  if (bt->split && c->split_sets) {
    Batch *hb[2];
    rc = split_halves(c, bt, hb);
    if (rc) return rc;
    *kernels = hb[0]->graph_kernels + hb[1]->graph_kernels;
    return 0;
  }
  rc = ensure_graph(bt, c->stream);
  if (rc) return rc;
  *kernels = bt->graph_kernels;
  return 0;
}

}  // extern "C"

// ============================================================================
// Output-time diagnostics (main.F90:202-216): GlobalQuantities, CalcStats,
// CalcDissipationNu and SlabDumper.  One kernel computes the per-plane sums
// and extrema of all of them; the host adds the chunks of each plane and the
// planes in a fixed order, so results do not depend on scheduling.
// ============================================================================
namespace {

int ensure_out(HostBox *hb, size_t doubles) {
  if (hb->out_doubles >= doubles) return 0;
  cudaFree(hb->d_out);
  hb->d_out = nullptr;
  hb->out_doubles = 0;
  if (cudaMalloc(&hb->d_out, doubles * sizeof(double)) != cudaSuccess)
    return fail(AFID_ENOMEM, "diagnostics staging of %zu doubles", doubles);
  hb->out_doubles = doubles;
  return 0;
}

// per-plane sums (q < PQ_NSUM) and extrema of box id, pl[k * PQ_N + q]
int plane_sums(afid_ctx *c, int id, HostBox **phb, std::vector<double> &pl) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (!rc) rc = set_device(c);
  if (rc) return rc;
  const int nxm = hb->dev.nxm;
  const size_t n = (size_t)nxm * PS_CHUNKS * PQ_N;
  rc = ensure_out(hb, n);
  if (rc) return rc;
  k_plane_sums<<<dim3(PS_CHUNKS, nxm), 256, 0, c->stream>>>(hb->d_self, hb->d_out);
  CKL();
  std::vector<double> raw(n);
  CK(cudaMemcpyAsync(raw.data(), hb->d_out, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  pl.assign((size_t)nxm * PQ_N, 0.0);
  for (int k = 0; k < nxm; ++k)
    for (int q = 0; q < PQ_N; ++q) {
      double v = raw[((size_t)k * PS_CHUNKS) * PQ_N + q];
      for (int ch = 1; ch < PS_CHUNKS; ++ch) {
        const double u = raw[((size_t)k * PS_CHUNKS + ch) * PQ_N + q];
        v = q < PQ_NSUM ? v + u : std::max(v, u);
      }
      pl[(size_t)k * PQ_N + q] = v;
    }
  *phb = hb;
  return 0;
}

}  // namespace

extern "C" int afid_global_quantities(afid_ctx *c, int id, afid_global_q *out) {
  if (!out) return fail(AFID_EINVAL, "null output");
  HostBox *hb;
  std::vector<double> pl;
  int rc = plane_sums(c, id, &hb, pl);
  if (rc) return rc;
  const afid_box_params &p = hb->prm;
  const int nxm = p.nxm;
  const double *xc = hb->xc.data();
  const double dx = (double)nxm / p.alx3;
  double anusin = 0, tempm = 0, vxr = 0, vyr = 0, vzr = 0, vall = 0;
  double vmz = 0, vmy = 0, vmx = 0, tmax = -1.7976931348623157e308, tmin = 1.7976931348623157e308;
  for (int k = 0; k < nxm; ++k) {
    // fac2 = g3rc(kc) (CreateGrid.F90:143-150)
    const double fac2 = k == 0 ? (xc[1] - xc[0]) * dx : (xc[k + 1] - xc[k - 1]) * dx * 0.5;
    const double *q = &pl[(size_t)k * PQ_N];
    anusin += q[PQ_TCVXC] * fac2;
    tempm += q[PQ_TC] * fac2;
    vxr += q[PQ_VX2] * fac2;
    vyr += q[PQ_VY2] * fac2;
    vzr += q[PQ_VZ2] * fac2;
    vall += (q[PQ_VZ2] + q[PQ_VY2] + q[PQ_VX2]) * fac2;
    vmz = std::max(vmz, q[PQ_MAXVZ]);
    vmy = std::max(vmy, q[PQ_MAXVY]);
    vmx = std::max(vmx, q[PQ_MAXVX]);
    tmax = std::max(tmax, q[PQ_MAXT]);
    tmin = std::min(tmin, -q[PQ_NEGMINT]);
  }
  const double vol = 1.0 / (p.alx3 * dx * (double)p.nzm * (double)p.nym);
  const double rradpr = std::sqrt(p.ray / p.pra);
  out->nu_vol = 1.0 + std::sqrt(p.pra * p.ray) * anusin * vol;
  out->vmax[0] = vmz;
  out->vmax[1] = vmy;
  out->vmax[2] = vmx;
  out->tempm = tempm * vol;
  out->tempmax = tmax;
  out->tempmin = tmin;
  out->vz_rms = std::sqrt(vzr * vol) * rradpr;
  out->vy_rms = std::sqrt(vyr * vol) * rradpr;
  out->vx_rms = std::sqrt(vxr * vol) * rradpr;
  out->vel_rms = std::sqrt(vall * vol) * rradpr;
  return 0;
}

extern "C" int afid_calc_stats(afid_ctx *c, int id) {
  HostBox *hb;
  std::vector<double> pl;
  int rc = plane_sums(c, id, &hb, pl);
  if (rc) return rc;
  const int nxm = hb->prm.nxm;
  const double usnym = 1.0 / hb->prm.nym, usnzm = 1.0 / hb->prm.nzm;
  static const int src[9] = {PQ_VX, PQ_VY, PQ_VZ, PQ_T, PQ_VX2, PQ_VY2, PQ_VZ2, PQ_T2, PQ_TVX};
  for (int a = 0; a < 9; ++a)
    for (int k = 0; k < nxm; ++k) hb->stats[(size_t)a * nxm + k] += pl[(size_t)k * PQ_N + src[a]] * usnzm * usnym;
  hb->nstatsamples += 1;
  return 0;
}

extern "C" int afid_calc_dissipation_nu(afid_ctx *c, int id, double *nu_mu, double *nu_th) {
  if (!nu_mu || !nu_th) return fail(AFID_EINVAL, "null output");
  HostBox *hb;
  std::vector<double> pl;
  int rc = plane_sums(c, id, &hb, pl);
  if (rc) return rc;
  const afid_box_params &p = hb->prm;
  const int nxm = p.nxm;
  const double *xc = hb->xc.data();
  const double dx = (double)nxm / p.alx3;
  const double ren = std::sqrt(p.ray / p.pra), pec = std::sqrt(p.pra * p.ray);
  auto xm = [&](int k) { return (xc[k] + xc[k + 1]) * 0.5; };
  double mu = 0.0, th = 0.0;
  for (int k = 0; k < nxm; ++k) {
    // lem, lec of CalcDissipationNu.F90:32-40
    const double lem = (xc[k + 1] - xc[k]) * dx;
    const double lec = k < nxm - 1 ? (xm(k + 1) - xm(k)) * dx : (xm(nxm - 1) - xm(nxm - 2)) * dx;
    const double *q = &pl[(size_t)k * PQ_N];
    mu += q[PQ_DISSTE] * lem * p.pra + q[PQ_DISSTE2] * lec * p.pra;
    th += q[PQ_DISSTH] * lem;
    hb->stats[(size_t)AFID_STAT_DISSTE * nxm + k] +=
        (q[PQ_DISSTE] + q[PQ_DISSTE2]) / (ren * (double)p.nym * (double)p.nzm);
    hb->stats[(size_t)AFID_STAT_DISSTH * nxm + k] += q[PQ_DISSTH] / (pec * (double)p.nym * (double)p.nzm);
  }
  const double volt = 1.0 / ((double)nxm * (double)p.nzm * (double)p.nym);
  *nu_mu = mu * volt + 1.0;
  *nu_th = th * volt;
  return 0;
}

extern "C" int afid_box_get_stats(afid_ctx *c, int id, double *out, int *nsamples) {
  if (!c || !out) return fail(AFID_EINVAL, "null argument");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  std::copy(hb->stats.begin(), hb->stats.end(), out);
  if (nsamples) *nsamples = hb->nstatsamples;
  return 0;
}

extern "C" int afid_box_reset_stats(afid_ctx *c, int id) {
  if (!c) return fail(AFID_EINVAL, "null ctx");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (rc) return rc;
  std::fill(hb->stats.begin(), hb->stats.end(), 0.0);
  hb->nstatsamples = 0;
  return 0;
}

extern "C" int afid_slab_locations(int nxm, const double *xc, const double *xslab, int *kslab) {
  if (!xc || !xslab || !kslab || nxm < 3) return fail(AFID_EINVAL, "slab_locations: bad argument");
  // InitializeSlabDump (SlabDumpRoutines.F90:52-67): kslab(1) = 2; slab m
  // = 2..9 at the last k in 2..nxm with xm(k-1) < xslab(m) < xm(k)
  auto xm = [&](int k1) { return (xc[k1 - 1] + xc[k1]) * 0.5; };   // 1-based xm(k)
  for (int m = 0; m < 9; ++m) kslab[m] = 2;
  for (int k = 2; k <= nxm; ++k)
    for (int m = 2; m <= 9; ++m)
      if (xm(k) > xslab[m - 2] && xm(k - 1) < xslab[m - 2]) kslab[m - 1] = k;
  return 0;
}

extern "C" int afid_slab_dump(afid_ctx *c, int id, const int *kslab, int nslab, double *out) {
  if (!c || !kslab || !out || nslab < 1 || nslab > 16) return fail(AFID_EINVAL, "slab_dump: 1..16 slabs");
  HostBox *hb;
  int rc = get_box(c, id, &hb);
  if (!rc) rc = set_device(c);
  if (rc) return rc;
  SlabList sl;
  for (int m = 0; m < nslab; ++m) {
    if (kslab[m] < 1 || kslab[m] > hb->prm.nxm)
      return fail(AFID_EINVAL, "slab_dump: kslab %d outside 1..nxm", kslab[m]);
    sl.k[m] = kslab[m] - 1;
  }
  const long long P = hb->dev.plane;
  const size_t n = (size_t)nslab * 4 * P;
  rc = ensure_out(hb, n);
  if (rc) return rc;
  k_slab_gather<<<dim3((unsigned)std::min<long long>(cdiv(P, 256), 1024), nslab), 256, 0, c->stream>>>(
      hb->d_self, sl, nslab, hb->d_out);
  CKL();
  CK(cudaMemcpyAsync(out, hb->d_out, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// ============================================================================
// Pressure solve without allocation.
//
// For callers that cannot allocate device memory at run time -- an
// application that hands all GPU memory to its own pool before it calls us,
// code that runs where cudaMalloc is not allowed, or a host program that
// keeps its fields on the device and must not grow its footprint per call --
// this entry point runs the same five pressure-solve kernels as
// afid_solve_pressure_correction, but keeps its scratch (half spectrum,
// Thomas pivots, metric tables, twiddles and kernel descriptors) in one
// file-scope device array instead of a box.  The caller passes only dph.
//
// The array is fixed at AFID_NOALLOC_DOUBLES doubles (about 48.5 MiB) and
// every GPU on which the library is loaded holds it until the process exits.
// Every call shares it and it keeps the previous call's contents; each call
// rewrites everything it reads (the status word is cleared by each call),
// so nothing has to start at zero.  Calls whose work overlaps on the GPU
// (two streams, or two host threads) race on it and must be serialised by
// the caller.  A call stages its small per-call data (tables, descriptor,
// status word) through host memory that the next call reuses, so a call on
// a stream that is being captured into a graph is refused.
// ============================================================================
namespace {

constexpr long long NOALLOC_MAX_SPEC = 1LL << 21;            // nxm * nzm * (nym/2 + 1)
constexpr int NOALLOC_MAX_NXM = 1024;
constexpr int NOALLOC_MAX_NYZ = AFID_MAX_NYZ;
constexpr long long NOALLOC_META = 1LL << 16;                // tables, twiddles, descriptors
constexpr long long AFID_NOALLOC_DOUBLES = 3 * NOALLOC_MAX_SPEC + NOALLOC_META;

static __device__ __align__(256) double g_noalloc_scratch[AFID_NOALLOC_DOUBLES];

// device address of g_noalloc_scratch per device (host code may not use the
// symbol itself as an address)
double *g_noalloc_base[64] = {};

int noalloc_setup(int dev) {
  if (dev < 0 || dev >= 64) return fail(AFID_EINVAL, "noalloc: device %d out of range", dev);
  if (g_noalloc_base[dev]) return 0;
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return fail(AFID_ECUDA, "noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
  g_noalloc_base[dev] = (double *)p;
  return 0;
}

// host staging of the small per-call data (no heap allocation per call)
struct NoallocHost {
  double tab[(size_t)T_NK * (NOALLOC_MAX_NXM + 1) + 2 * NOALLOC_MAX_NYZ];
  double2 tw[2 * NOALLOC_MAX_NYZ];
  CUtensorMap tm;
};
NoallocHost g_noalloc_host;

}  // namespace

extern "C" int afid_solve_pressure_correction_noalloc(double *dph, int nxm, int nym, int nzm,
                                                      const double *xc, double alx3, double ylen,
                                                      double zlen, void *stream, int *status) {
  if (!dph || !xc) return fail(AFID_EINVAL, "noalloc: dph and xc are required");
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const cudaError_t e = cudaStreamIsCapturing((cudaStream_t)stream, &cs);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(AFID_EINVAL, "noalloc: the stream's capture state cannot be read (%s)", cudaGetErrorString(e));
    }
    if (cs != cudaStreamCaptureStatusNone)
      return fail(AFID_EINVAL, "noalloc: the stream is being captured; this entry point stages per-call data "
                               "through host memory and cannot be recorded into a graph");
  }
  if (nxm < 3 || nym < 2 || nzm < 2 || (nym % 2))
    return fail(AFID_EINVAL, "noalloc: need nxm >= 3, nzm >= 2 and an even nym >= 2");
  if (!(alx3 > 0) || !(ylen > 0) || !(zlen > 0)) return fail(AFID_EINVAL, "noalloc: lengths must be > 0");
  const long long nspec = (long long)nxm * nzm * (nym / 2 + 1);
  if (nxm > NOALLOC_MAX_NXM || nym > NOALLOC_MAX_NYZ || nzm > NOALLOC_MAX_NYZ || nspec > NOALLOC_MAX_SPEC)
    return fail(AFID_ESIZE,
                "noalloc: box %dx%dx%d exceeds the fixed scratch: nxm <= %d, nym, nzm <= %d and "
                "nxm*nzm*(nym/2+1) <= %lld (got %lld)",
                nxm, nym, nzm, NOALLOC_MAX_NXM, NOALLOC_MAX_NYZ, NOALLOC_MAX_SPEC, nspec);
  if ((uintptr_t)dph & 15) return fail(AFID_EINVAL, "noalloc: dph must be 16-byte aligned");
  for (int k = 1; k <= nxm; ++k)
    if (!(xc[k] > xc[k - 1])) return fail(AFID_EINVAL, "noalloc: xc must be increasing");
  BoxDev d;
  memset(&d, 0, sizeof d);
  if (factor_radices(nym, d.fft_y_radix, &d.fft_y_np) || factor_radices(nzm, d.fft_z_radix, &d.fft_z_np))
    return fail(AFID_EFFT, "noalloc: nym=%d nzm=%d need prime factors <= 7", nym, nzm);
  if (!warp_plan(nym, &d.wy_v, &d.wy_g, d.wy_rad, &d.wy_np, 2)) d.wy_v = 0;
  if (!warp_plan(nzm, &d.wz_v, &d.wz_g, d.wz_rad, &d.wz_np)) d.wz_v = 0;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  int rc = noalloc_setup(dev);
  if (rc) return rc;
  rc = init_kernel_attrs();
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  double *base = g_noalloc_base[dev];

  // device layout of the scratch array (offsets in doubles)
  const int nx = nxm + 1;
  const long long o_spec = 0, o_dstore = 2 * NOALLOC_MAX_SPEC, o_meta = 3 * NOALLOC_MAX_SPEC;
  const long long n_tab = (long long)T_NK * nx + nzm + nym;
  const long long o_tab = o_meta;
  const long long o_tw = (o_tab + n_tab + 1) & ~1LL;
  const long long o_sc = (o_tw + 2LL * (nym + nzm) + 7) & ~7LL;
  const long long o_box = o_sc + (long long)((sizeof(BoxScalars) + 63) / 8);
  const long long o_off = o_box + (long long)((sizeof(BoxDev) + 63) / 8);
  const long long o_tm = (o_off + 16 + 7) & ~7LL;   // 64-byte aligned TMA map of the z transform
  if (o_tm + 16 > AFID_NOALLOC_DOUBLES) return fail(AFID_ESIZE, "noalloc: tables do not fit");

  // tables: the Poisson rows of InitPressureSolver.F90:22-59 (other k-tables unused)
  double *tab = g_noalloc_host.tab;
  for (long long q = 0; q < n_tab; ++q) tab[q] = 0.0;
  {
    const double pi = 2.0 * std::asin(1.0);
    const double dx = (double)nxm / alx3, dxq = dx * dx;
    auto g3rm = [&](int kc) { return (xc[kc] - xc[kc - 1]) * dx; };               // kc 1-based
    auto g3rc = [&](int kc) {
      if (kc == 1) return (xc[1] - xc[0]) * dx;
      if (kc == nx) return (xc[nx - 1] - xc[nxm - 1]) * dx;
      return (xc[kc] - xc[kc - 2]) * dx * 0.5;
    };
    for (int kc = 1; kc <= nxm; ++kc) {
      const int kp = (kc == nxm) ? kc : kc + 1;
      const double kmc = (kc == 1) ? 0.0 : 1.0, kpc = (kc == nxm) ? 0.0 : 1.0;
      const double a33icc = kmc * dxq / g3rc(kc);
      const double a33icp = kpc * dxq / g3rc(kp);
      const double ugmmm = 1.0 / g3rm(kc);
      tab[(size_t)T_AMPHK * nx + kc - 1] = a33icc * ugmmm;
      tab[(size_t)T_APPHK * nx + kc - 1] = a33icp * ugmmm;
      tab[(size_t)T_ACPHK * nx + kc - 1] = -(a33icc * ugmmm + a33icp * ugmmm);
    }
    double *ak1 = tab + (size_t)T_NK * nx, *ak2 = ak1 + nzm;
    const int nzmh = nzm / 2 + 1, nymh = nym / 2 + 1;
    for (int i = 1; i <= nzm; ++i) {
      const double ao = (i <= nzmh) ? (i - 1) * 2.0 * pi : -(nzm - i + 1) * 2.0 * pi;
      const double f = (double)nzm / zlen;
      ak1[i - 1] = 2.0 * (1.0 - std::cos(ao / nzm)) * (f * f);
    }
    for (int j = 1; j <= nym; ++j) {
      const double ap = (j <= nymh) ? (j - 1) * 2.0 * pi : -(nym - j + 1) * 2.0 * pi;
      const double f = (double)nym / ylen;
      ak2[j - 1] = 2.0 * (1.0 - std::cos(ap / nym)) * (f * f);
    }
  }
  build_twiddles(nym, g_noalloc_host.tw);
  build_twiddles(nzm, g_noalloc_host.tw + nym);

  // descriptor of a one-box batch pointing into the scratch array; dph is
  // both the input (phi) and the output of the solve
  d.nxm = nxm; d.nx = nx; d.nym = nym; d.nzm = nzm; d.nymh = nym / 2 + 1;
  d.nsst = 1;
  d.plane = (long long)nym * nzm;
  d.fsize = (long long)nx * d.plane;
  d.nspec = nspec;
  d.phi = dph;
  d.spec = (double2 *)(base + o_spec);
  d.dstore = base + o_dstore;
  d.tab = base + o_tab;
  d.twy = (const double2 *)(base + o_tw);
  d.twz = (const double2 *)(base + o_tw) + nym;
  d.sc = (BoxScalars *)(base + o_sc);
  d.tm_z = (const CUtensorMap *)(base + o_tm);
  d.active = 1;
  d.piv_ready = 1;   // k_poisson_pivots runs first in every call
  rc = encode_z_map(d, &g_noalloc_host.tm);
  if (rc) return rc;
  BoxScalars bs;
  memset(&bs, 0, sizeof bs);
  // one-box tile tables of every family (only the transforms' and the
  // x-solve's are used)
  int off[NFAM][2], total[NFAM];
  static_assert(sizeof(off) <= 16 * sizeof(double), "tile tables exceed their scratch slot");
  for (int f = 0; f < NFAM; ++f) {
    off[f][0] = 0;
    off[f][1] = total[f] = (f == FAM_FY || f == FAM_FZ || f == FAM_PX || f >= FAM_WY8) ? (int)tiles_of(d, f) : 0;
  }
  CK(cudaMemcpyAsync(base + o_tab, tab, (size_t)n_tab * 8, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_tw, g_noalloc_host.tw, (size_t)(nym + nzm) * 16, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_sc, &bs, sizeof bs, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_box, &d, sizeof d, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_off, off, sizeof off, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_tm, &g_noalloc_host.tm, sizeof(CUtensorMap), cudaMemcpyHostToDevice, st));
  const BoxDev *dbox = (const BoxDev *)(base + o_box);
  const int *doff = (const int *)(base + o_off);
  auto bd = [&](int fam) { return BatchDev{dbox, doff + 2 * fam, 1}; };
  FftSmem smy{0, 0}, smz{0, 0};
  int twy = 0, twz = 0, gy = 0, gz = 0;
  fft_smem_grow(d, smy, smz, twy, twz);
  const size_t sy = (size_t)(2 * smy.slot + twy) * 16 + FFT_TAIL_BYTES;
  const size_t sz = (size_t)(2 * smz.slot + twz) * 16 + FFT_TAIL_BYTES;
  size_t swy[WY_NV];
  int gwy[WY_NV], gwz[WY_NV];
  rc = fft_grid(k_fft_y_fwd, sy, total[FAM_FY], &gy);
  if (!rc) rc = fft_grid(k_fft_z<-1>, sz, total[FAM_FZ], &gz);
  if (!rc) rc = wy_shapes(std::vector<BoxDev>{d}, total, swy, gwy, gwz);
  if (rc) return rc;
  // the x-solve's pivots, for this call's grid
  k_poisson_pivots<<<(unsigned)cdiv(px_pairs(nzm, d.nymh), 256), 256, 0, st>>>(d);
  CKL();
  rc = launch_fft_y(true, total, bd, gy, sy, smy, gwy, swy, st, 0);
  if (rc) return rc;
  rc = launch_fft_z<-1>(total, bd, gz, sz, smz, gwz, swy, st, 0);
  if (rc) return rc;
  rc = launch_poisson_x(total, bd, st, 0);
  if (rc) return rc;
  rc = launch_fft_z<+1>(total, bd, gz, sz, smz, gwz, swy, st, 0);
  if (rc) return rc;
  rc = launch_fft_y(false, total, bd, gy, sy, smy, gwy, swy, st, 0);
  if (rc) return rc;
  if (status) {
    // wait for this call's kernels and report its status word
    int v = -1;
    CK(cudaMemcpyAsync(&v, (char *)(base + o_sc) + offsetof(BoxScalars, status), sizeof v,
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *status = v;
  }
  return 0;
}
