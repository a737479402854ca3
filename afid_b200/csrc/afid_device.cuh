// Device-side data structures shared by every kernel of the AFiD RK3 path.
//
// Field layout in HBM ("plane-major"): a 3-D field q(k, j, i) of the
// reference (x = wall-normal k, periodic y = j, periodic z = i; Fortran
// order k fastest) is stored as q[k][i][j], i.e. y fastest, then z, then x.
//   * the x-tridiagonal solves run one thread per (j, i) column and march k,
//     so a warp reads 32 consecutive j: coalesced;
//   * the y-FFT reads contiguous y-rows;
//   * the z-FFT reads tiles of consecutive ky for every kz;
//   * the explicit stencils march k with a (y, z) tile in shared memory and
//     keep the x-neighbours of their own column in a ring of planes.
// There is no halo storage: periodic neighbours are index wraps.
#pragma once
#include <cuda.h>            // CUtensorMap
#include <cuda_runtime.h>
#include <stdint.h>

namespace afid {

// Per-box scalars that live on the device so that dt can be chosen on the
// device (CFL rule) and a whole step can be captured in a CUDA graph.
struct BoxScalars {
  double dt;        // current time step
  double time;      // simulation time
  double al, ga, ro, beta;   // current substep coefficients, beta = dt/(2 Re)
  double cfl;       // max CFL number of the current velocity (CalcMaxCFL)
  double cfl_used;  // cfl*dt (fixed dt) or cfl (variable dt), main.F90:171-189
  double divmax;    // max |div u| (CheckDivergence, without 1/(al dt))
  double vmax[3];   // max |vz|, |vy|, |vx| (GlobalQuantities vmax order)
  double nu_bot, nu_top;     // plate Nusselt numbers (CalcPlateNu)
  // dt policy (bou.in)
  double cflmax, dtmin, dtmax, limitvel, resid;
  int idtv;         // 1 = variable dt
  int ntime;        // step counter (main.F90 ntime)
  int status;       // 0 ok, else the reference's error code (165/166/169/266)
  int nonfinite;    // set when a non-finite value is seen by the diagnostics
  unsigned long long red_u64[4];  // atomicMax scratch: cfl, div, vmax_y, vmax_z
  double nu_partial_dummy;
  // holds (afid_box_set_stop): after a step the box is put on hold (status
  // AFID_STATUS_HELD) when ntime reaches stop_ntime (> 0), with tout > 0 at
  // an output time of main.F90:207 (second step, or mod(time, tout) < dt),
  // and with tmax > 0 once time > tmax (main.F90:256)
  double tout;
  double tmax;
  int stop_ntime;
  int pad_hold_;
};

// status of a box on hold: skipped like a failed box until resumed
constexpr int AFID_STATUS_HELD_DEV = 1;

// Offsets of the metric tables inside BoxDev::tab (length nx each unless
// noted).  Index k is 0-based (k = kc-1 of the reference).
enum TabId {
  T_UDX3C = 0, T_UDX3M, T_AM3CK, T_AC3CK, T_AP3CK, T_AM3SK, T_AC3SK, T_AP3SK,
  T_AM3SSK, T_AC3SSK, T_AP3SSK, T_AMPHK, T_ACPHK, T_APPHK, T_XC, T_G3RC,
  T_G3RM, T_NK  // number of k-tables
};

// Per-substep tridiagonal tables in BoxDev::coef: for system s in
// {SYS_X (vx, size nx), SYS_YZ (vy/vz, size nxm), SYS_T (temp, size nx)}
// the arrays (sc, fact, dp, du, g) each of length nx at
// coef[(s * C_N + a) * nx + k].
enum SysId { SYS_X = 0, SYS_YZ = 1, SYS_T = 2, SYS_N = 3 };
enum CoefId { C_SC = 0, C_FACT, C_DP, C_DU, C_G, C_N };

constexpr int HIST_FIELDS = 8;   // time, dt, cfl_used, divmax, nu_bot, nu_top, vmax_y, vmax_z

struct BoxDev {
  int nx, nxm, nym, nzm, nymh;
  int nsst;
  int inslws, inslwn;
  long long plane;      // nym * nzm
  long long fsize;      // nx * plane
  long long nspec;      // nxm * nzm * nymh
  double dx, dy, dz, dxq, dyq, dzq, ren, pec, tempbp, temptp;
  double inv_nyz;       // unused by kernels; kept for diagnostics
  // prognostic fields, nx planes each
  double *vx, *vy, *vz, *temp, *pr;
  // RK history (H of the previous substep)
  double *rux, *ruy, *ruz, *rutemp;
  // the reference's rhs(1, :, :) row, carried between implicit solves
  double *wall;
  // forward-sweep intermediates of the four implicit solves (scratch)
  double *ybuf[4];
  // Poisson scratch (aliases ybuf storage; live only between the divergence
  // and the correction)
  double2 *spec;        // [k][kz][ky], k < nxm, ky <= nym/2
  double *dstore;       // reciprocal Thomas pivots 1/d of the Poisson solve,
                        // same indexing (tabulated by k_poisson_pivots)
  double *phi;          // pressure correction dph, [k][i][j], k < nxm
  // reference-boundary mode buffers (allocated on first use)
  double *qcap, *dq, *hro, *rhs;
  // tables
  const double *tab;    // T_NK*nx k-tables, then ak1[nzm], ak2[nym]
  const double2 *twy;   // exp(-2 pi i n / nym), n < nym
  const double2 *twz;   // exp(-2 pi i n / nzm), n < nzm
  double *coef;         // per-substep tridiagonal tables
  double *nu_part;      // per-block partial sums of the plate Nu reduction
  double *hist;         // per-step records, HIST_FIELDS doubles each (ring)
  int hist_cap;
  int pad1_;
  BoxScalars *sc;
  int fft_y_radix[16];  // radices of nym (Stockham passes), terminated by 0
  int fft_z_radix[16];  // radices of nzm
  int fft_y_np, fft_z_np;
  int active;           // 0 = skipped by every kernel
  int k1_minb;          // tuning: variant of the explicit/forward kernel (2, 3 or 4)
  int fy_lines;         // tuning: row pairs per y-FFT block (0 = default)
  int fz_lines;         // tuning: ky columns per z-FFT block (0 = default)
  int fz_rb;            // kz rows per TMA box of the z transform (a divisor of nzm, <= 256)
  const CUtensorMap *tm_z;  // TMA map of spec as a 2-D FP64 array (2*nymh x nxm*nzm), box 2L x fz_rb
  int piv_ready;        // 1 = dstore holds the Poisson pivots of this grid
  // warp-transform plan of the y transforms (k_fftw.cuh): wy_v values per
  // lane (0: no plan, the tile kernels run), wy_g lanes per line, radices
  int wy_v, wy_g, wy_np;
  int wy_rad[8];
  // the same for the z transforms (k_fftw_z): 0 = the tile kernel runs
  int wz_v, wz_g, wz_np;
  int wz_rad[8];
  // test switch of the bounded waits (afid_box_test_skip_z_copies): the z
  // transform arms its slot mbarriers without issuing the box's tile copies,
  // and its waits give up after mbar_tries polls (0: MBAR_MAX_TRIES)
  int z_copy_skip;
  unsigned mbar_tries;
};

// Work decomposition: each kernel family launches a 1-D grid over the
// concatenated tiles of all boxes of a batch.  tile_off[b] is the first
// block of box b, tile_off[nbox] the total.
struct BatchDev {
  const BoxDev *boxes;
  const int *tile_off;  // [nbox + 1] for this kernel family
  int nbox;
};

__device__ __forceinline__ int find_box(const int *off, int nbox, int blk) {
  int lo = 0, hi = nbox - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= blk) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ double tabk(const BoxDev &B, int t, int k) {
  return __ldg(B.tab + (long long)t * B.nx + k);
}

__device__ __forceinline__ int wrap(int a, int n) {
  return a < 0 ? a + n : (a >= n ? a - n : a);
}

// Complex helpers (double2 = re, im).
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// Order-preserving map of a non-negative double onto uint64 for atomicMax.
__device__ __forceinline__ unsigned long long dbits(double v) {
  return (unsigned long long)__double_as_longlong(v);
}

// Asynchronous global -> shared copies (cp.async): 16 bytes bypassing L1,
// 8 bytes through L1; groups are committed and waited for explicitly.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(src));
}
__device__ __forceinline__ void cp_async8d(void *dst, const void *src) {
  unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(saddr), "l"(src));
}
__device__ __forceinline__ void cp_async8(double *dst, const double *src) { cp_async8d(dst, src); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_commit_wait() {
  cp_async_commit();
  cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// TMA (cp.async.bulk.tensor) loads into shared memory, completed on an
// mbarrier.  Waits are bounded: after MBAR_MAX_TRIES polls the caller treats
// the copy as failed (status AFID_STATUS_DEVICE_TIMEOUT) instead of spinning.
// ---------------------------------------------------------------------------
constexpr unsigned MBAR_MAX_TRIES = 1u << 22;
constexpr int AFID_STATUS_DEVICE_TIMEOUT = 990;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// order this thread's generic-proxy shared-memory accesses before later
// async-proxy (TMA) accesses
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity,
                                                  unsigned tries = MBAR_MAX_TRIES) {
  for (unsigned t = 0; t < tries; ++t)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// 1-D bulk copy of ``bytes`` (a multiple of 16) from global src to shared
// dst, both 16-byte aligned, completed on ``bar``
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// 2-D tile load of box (x, y) of ``map`` into shared memory at dst (16-byte
// aligned); x times the element size must be a multiple of 16 bytes
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, unsigned long long *bar, int x,
                                            int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
      "[%2];\n" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

}  // namespace afid
