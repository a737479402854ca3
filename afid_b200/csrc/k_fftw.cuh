// Warp transforms along y (the r2c and c2r steps of
// SolvePressureCorrection.F90:97 and :148) and along z (the c2c steps of
// SolvePressureCorrection.F90:102 and :141).
//
// Each warp transforms LPW = 32 / G complex lines of length N on its own:
// G lanes per line, V = N / G values per lane (8 or 12).  The plan is a mixed-radix
// Stockham sequence whose radices all divide V, so in every pass each lane
// computes exactly V / R butterflies of radix R (no idle lanes).  Passes
// exchange data through the warp's own shared-memory region (LPW lines x N
// values, interleaved n * LPW + line) with __syncwarp only: warps never wait
// for each other.  The first pass of the forward transform loads its
// butterflies' inputs straight from HBM (two real rows per complex line, the
// lanes of a line reading consecutive values); the last pass of the inverse
// transform stores straight to HBM.
//
// Warps are independent: a warp unit is LPW lines (2 LPW rows of one plane)
// of one box, the units of a launch are numbered across its boxes, and each
// warp of the (persistent) grid takes runs of WF_RUN consecutive units,
// the runs dealt round-robin over all warps.  A warp keeps the fields of its
// current box in registers and that box's twiddles and radices in its own
// slice of shared memory, reloading them (with __syncwarp only) when its
// unit belongs to another box: a block has no barrier at all.
#pragma once
#include "k_fft.cuh"

namespace afid {

constexpr int WF_WARPS = 8;            // warps per block
constexpr int WF_T = 32 * WF_WARPS;    // threads per block
constexpr int WF_RUN = 4;              // consecutive units per run of a warp
constexpr int WF_MAX_N = 128;          // longest line with a warp plan

// lines per warp and units per plane of box B's y plan
__host__ __device__ __forceinline__ int wy_lpw(const BoxDev &B) { return 32 / B.wy_g; }
__host__ __device__ __forceinline__ int wy_units_per_plane(const BoxDev &B) {
  return (B.nzm + 2 * wy_lpw(B) - 1) / (2 * wy_lpw(B));
}
// the same for the z plan: a unit is LPW neighbouring ky columns of a plane
__host__ __device__ __forceinline__ int wz_lpw(const BoxDev &B) { return 32 / B.wz_g; }
__host__ __device__ __forceinline__ int wz_units_per_plane(const BoxDev &B) {
  return (B.nymh + wz_lpw(B) - 1) / wz_lpw(B);
}

// a warp's slice of shared memory: twiddles (WF_MAX_N complex), radices
// (8 ints, 32 bytes), then the work region (32 V complex)
__host__ __device__ __forceinline__ int wf_slice(int V) { return WF_MAX_N + 2 + 32 * V; }   // complex values
__host__ __device__ __forceinline__ size_t wf_smem_bytes(int V) { return (size_t)WF_WARPS * wf_slice(V) * 16; }

// The unit sequence of a warp: runs gw, gw + W, gw + 2W, ... of WF_RUN
// units (gw: the warp's index in the grid, W: the grid's warps).
struct WarpUnits {
  int gw, nw, total;
  __device__ __forceinline__ explicit WarpUnits(int total_)
      : gw((int)(blockIdx.x * WF_WARPS + (threadIdx.x >> 5))), nw((int)(gridDim.x * WF_WARPS)), total(total_) {}
  __device__ __forceinline__ int first() const { return gw * WF_RUN < total ? gw * WF_RUN : total; }
  __device__ __forceinline__ int next(int u) const {
    int n = u + 1;
    if (n % WF_RUN == 0) n = (u / WF_RUN + nw) * WF_RUN;
    return n < total ? n : total;
  }
};

// The fields of a box a warp transform needs, held in registers; load()
// also copies the box's twiddles and radices into the warp's slice.  ZDIR
// selects the z plan: lines of nzm points, LPW columns per unit.
template <bool ZDIR = false>
struct WarpBox {
  int b, N, nzm, nh, nxm, lpw, lgL, upp, np;
  long long plane;
  double *phi;
  double2 *spec;
  bool run;
  __device__ __forceinline__ void load(const BatchDev &bt, int bi, int ns, double2 *tws, int *rad) {
    const BoxDev *Bp = bt.boxes + bi;
    b = bi;
    nzm = __ldg(&Bp->nzm);
    nh = __ldg(&Bp->nymh);
    nxm = __ldg(&Bp->nxm);
    N = ZDIR ? nzm : __ldg(&Bp->nym);
    lpw = 32 / __ldg(ZDIR ? &Bp->wz_g : &Bp->wy_g);
    lgL = ilog2(lpw);
    upp = ZDIR ? (nh + lpw - 1) / lpw : (nzm + 2 * lpw - 1) / (2 * lpw);
    np = __ldg(ZDIR ? &Bp->wz_np : &Bp->wy_np);
    plane = __ldg(&Bp->plane);
    phi = (double *)__ldg((const unsigned long long *)&Bp->phi);
    spec = (double2 *)__ldg((const unsigned long long *)&Bp->spec);
    const double2 *tw = (const double2 *)__ldg((const unsigned long long *)(ZDIR ? &Bp->twz : &Bp->twy));
    run = __ldg(&Bp->active) && ns < __ldg(&Bp->nsst) &&
          *(volatile int *)&((BoxScalars *)__ldg((const unsigned long long *)&Bp->sc))->status == 0;
    const int lane = threadIdx.x & 31;
    for (int q = lane; q < N; q += 32) tws[q] = __ldg(tw + q);
    if (lane < 8) rad[lane] = __ldg(ZDIR ? &Bp->wz_rad[lane] : &Bp->wy_rad[lane]);
    __syncwarp();
  }
};

// One Stockham pass of radix R over the warp's LPW lines (lane: line
// lane % LPW, butterflies j = lane / LPW + b G for b < V / R).
template <int R, int SGN, int V, class Src, class Dst>
__device__ __forceinline__ void wpass(int N, int lgL, int Ns, const double2 *tw, const Src &src, const Dst &dst) {
  constexpr int BPT = V / R;
  const int lane = threadIdx.x & 31;
  const int NR = N / R, tstr = N / (Ns * R);
  const FastDiv dNs(Ns);
  const int l = lane & ((1 << lgL) - 1), j0 = lane >> lgL, jstep = 32 >> lgL;
  double2 v[BPT][R];
#pragma unroll
  for (int b = 0; b < BPT; ++b) {
    const int j = j0 + b * jstep;
#pragma unroll
    for (int r = 0; r < R; ++r) v[b][r] = src(l, j + r * NR);
  }
  __syncwarp();
#pragma unroll
  for (int b = 0; b < BPT; ++b) {
    const int j = j0 + b * jstep;
    const int k = dNs.mod(j);
    if (Ns > 1) twiddle<R, SGN>(v[b], k, tstr, tw);
    dft_small<R, SGN>(v[b], tw, N);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst(l, base + r * Ns, v[b][r]);
  }
  __syncwarp();
}

template <int SGN, int V, class Src, class Dst>
__device__ __forceinline__ void wrun(int R, int N, int lgL, int Ns, const double2 *tw, const Src &src, const Dst &dst) {
  // only the radices that divide V occur in a plan with V values per lane
  switch (R) {
    case 2: if constexpr (V % 2 == 0) wpass<2, SGN, V>(N, lgL, Ns, tw, src, dst); break;
    case 3: if constexpr (V % 3 == 0) wpass<3, SGN, V>(N, lgL, Ns, tw, src, dst); break;
    case 4: if constexpr (V % 4 == 0) wpass<4, SGN, V>(N, lgL, Ns, tw, src, dst); break;
    case 6: if constexpr (V % 6 == 0) wpass<6, SGN, V>(N, lgL, Ns, tw, src, dst); break;
    case 8: if constexpr (V % 8 == 0) wpass<8, SGN, V>(N, lgL, Ns, tw, src, dst); break;
    case 12: if constexpr (V % 12 == 0) wpass<12, SGN, V>(N, lgL, Ns, tw, src, dst); break;
    default: if constexpr (V % 16 == 0) wpass<16, SGN, V>(N, lgL, Ns, tw, src, dst); break;
  }
}

// The warp's whole transform: the first pass reads src, the last writes dst
// (the passes between go through the warp's region a).
template <int SGN, int V, class Src, class Dst>
__device__ __forceinline__ void wfft(double2 *a, int N, int lgL, const int *rad, int np, const double2 *tw,
                                     const Src &src, const Dst &dst) {
  const SmemSrc as{a, lgL};
  const SmemDst ad{a, lgL};
  if (np == 1) {
    wrun<SGN, V>(rad[0], N, lgL, 1, tw, src, dst);
    return;
  }
  wrun<SGN, V>(rad[0], N, lgL, 1, tw, src, ad);
  int Ns = rad[0];
  for (int p = 1; p < np - 1; ++p) {
    wrun<SGN, V>(rad[p], N, lgL, Ns, tw, as, ad);
    Ns *= rad[p];
  }
  wrun<SGN, V>(rad[np - 1], N, lgL, Ns, tw, as, dst);
}

// first pass of the forward transform: line p = rows (2p, 2p+1) of the
// unit, read from HBM (rows beyond nzm are zero)
struct WRowPairSrc {
  const double *rows;   // row 2p of line p at rows + 2 p N
  int N, nrow;          // rows present in the unit
  __device__ __forceinline__ double2 operator()(int p, int n) const {
    const double a = 2 * p < nrow ? __ldcg(rows + (long long)(2 * p) * N + n) : 0.0;
    const double b = 2 * p + 1 < nrow ? __ldcg(rows + (long long)(2 * p + 1) * N + n) : 0.0;
    return make_double2(a, b);
  }
};


// Forward (r2c) y transform of the units of the launch.
template <int V>
__global__ void __launch_bounds__(WF_T, 2) k_fftw_y_fwd(BatchDev bt, int ns, int total) {
  extern __shared__ double2 wsm[];
  double2 *const tws = wsm + (threadIdx.x >> 5) * wf_slice(V);   // this warp's slice
  int *const rad = reinterpret_cast<int *>(tws + WF_MAX_N);
  double2 *const reg = tws + WF_MAX_N + 2;
  const int lane = threadIdx.x & 31;
  const WarpUnits wu(total);
  if (wu.first() >= total) return;
  TileWalk wk(bt, wu.first());
  WarpBox<> X;
  X.b = -1;
  for (int u = wu.first(); u < total; u = wu.next(u)) {
    const int lu = wk.to(bt, u);
    if (wk.b != X.b) X.load(bt, wk.b, ns, tws, rad);
    if (!X.run) continue;
    const int N = X.N, lpw = X.lpw, lgL = X.lgL;
    const int k = lu / X.upp, i0 = (lu - k * X.upp) * 2 * lpw;
    const int nrow = min(2 * lpw, X.nzm - i0);
    const double *rows = X.phi + (long long)k * X.plane + (long long)i0 * N;
    wfft<-1, V>(reg, N, lgL, rad, X.np, tws, WRowPairSrc{rows, N, nrow}, SmemDst{reg, lgL});
    // unpack the two real transforms of line l: A = (Z_q + conj Z_{N-q}) / 2,
    // B = (Z_q - conj Z_{N-q}) / (2i), q <= N/2
    const int l = lane & (lpw - 1), g = 32 / lpw, nh = X.nh;
    double2 *const speck = X.spec + (long long)k * X.nzm * nh;
    const int i = i0 + 2 * l;
    for (int q = lane >> lgL; q < nh; q += g) {
      const double2 z = reg[sidx(l, q, lgL)];
      const double2 zn = reg[sidx(l, q == 0 ? 0 : N - q, lgL)];
      const double2 A = make_double2((z.x + zn.x) * 0.5, (z.y - zn.y) * 0.5);
      const double2 Bv = make_double2((z.y + zn.y) * 0.5, (zn.x - z.x) * 0.5);
      if (i < X.nzm) __stcg(speck + (long long)i * nh + q, A);
      if (i + 1 < X.nzm) __stcg(speck + (long long)(i + 1) * nh + q, Bv);
    }
    __syncwarp();
  }
}

// first pass of the inverse transform: line p = the complex line
// A + i B of the half-spectrum rows (2p, 2p+1), read from HBM with the
// Hermitian extension (the imaginary parts at ky = 0 and ky = N/2 ignored,
// as in a c2r transform)
struct WHalfPairSrc {
  const double2 *rows;  // row 2p of line p at rows + 2 p nh
  int N, nh, nrow;
  __device__ __forceinline__ double2 coef(int r, int n) const {
    if (r >= nrow) return make_double2(0.0, 0.0);
    const int q = n < nh ? n : N - n;
    double2 c = __ldcg(rows + (long long)r * nh + q);
    if (q == 0 || 2 * q == N) c.y = 0.0;
    else if (n >= nh) c.y = -c.y;
    return c;
  }
  __device__ __forceinline__ double2 operator()(int p, int n) const {
    const double2 A = coef(2 * p, n), Bv = coef(2 * p + 1, n);
    return make_double2(A.x - Bv.y, A.y + Bv.x);
  }
};
// last pass of the inverse transform: the real and imaginary parts are the
// two output rows, stored to HBM
struct WRowPairDst {
  double *rows;
  int N, nrow;
  __device__ __forceinline__ void operator()(int p, int n, double2 v) const {
    if (2 * p < nrow) __stcg(rows + (long long)(2 * p) * N + n, v.x);
    if (2 * p + 1 < nrow) __stcg(rows + (long long)(2 * p + 1) * N + n, v.y);
  }
};

// Inverse (c2r) y transform of the units of the launch.
template <int V>
__global__ void __launch_bounds__(WF_T, 2) k_fftw_y_inv(BatchDev bt, int ns, int total) {
  extern __shared__ double2 wsm[];
  double2 *const tws = wsm + (threadIdx.x >> 5) * wf_slice(V);
  int *const rad = reinterpret_cast<int *>(tws + WF_MAX_N);
  double2 *const reg = tws + WF_MAX_N + 2;
  const WarpUnits wu(total);
  if (wu.first() >= total) return;
  TileWalk wk(bt, wu.first());
  WarpBox<> X;
  X.b = -1;
  for (int u = wu.first(); u < total; u = wu.next(u)) {
    const int lu = wk.to(bt, u);
    if (wk.b != X.b) X.load(bt, wk.b, ns, tws, rad);
    if (!X.run) continue;
    const int N = X.N, lpw = X.lpw, lgL = X.lgL, nh = X.nh;
    const int k = lu / X.upp, i0 = (lu - k * X.upp) * 2 * lpw;
    const int nrow = min(2 * lpw, X.nzm - i0);
    const double2 *half = X.spec + (long long)k * X.nzm * nh + (long long)i0 * nh;
    double *rows = X.phi + (long long)k * X.plane + (long long)i0 * N;
    wfft<+1, V>(reg, N, lgL, rad, X.np, tws, WHalfPairSrc{half, N, nh, nrow}, WRowPairDst{rows, N, nrow});
  }
}

// z lines: column ky0 + l of one plane's spectrum (row pitch nh), read and
// written in place in HBM; columns at or beyond nh read as zero and are not
// stored.  Every value a warp's pass reads is read before any is written
// (wpass loads all its inputs ahead of a __syncwarp), so a single-pass plan
// is in place too.
struct WColSrc {
  const double2 *S;
  int nh, ky0;
  __device__ __forceinline__ double2 operator()(int l, int n) const {
    return ky0 + l < nh ? __ldcg(S + (long long)n * nh + ky0 + l) : make_double2(0.0, 0.0);
  }
};
struct WColDst {
  double2 *S;
  int nh, ky0;
  __device__ __forceinline__ void operator()(int l, int n, double2 v) const {
    if (ky0 + l < nh) __stcg(S + (long long)n * nh + ky0 + l, v);
  }
};

// c2c z transform (SGN -1 forward, +1 inverse) of the units of the launch:
// a unit is LPW neighbouring ky columns of one plane, so the lanes reading
// one kz row of the unit read LPW consecutive complex values, and the runs of
// units that neighbouring warps take cover neighbouring columns of the rows.
template <int SGN, int V>
__global__ void __launch_bounds__(WF_T, 2) k_fftw_z(BatchDev bt, int ns, int total) {
  extern __shared__ double2 wsm[];
  double2 *const tws = wsm + (threadIdx.x >> 5) * wf_slice(V);
  int *const rad = reinterpret_cast<int *>(tws + WF_MAX_N);
  double2 *const reg = tws + WF_MAX_N + 2;
  const WarpUnits wu(total);
  if (wu.first() >= total) return;
  TileWalk wk(bt, wu.first());
  WarpBox<true> X;
  X.b = -1;
  for (int u = wu.first(); u < total; u = wu.next(u)) {
    const int lu = wk.to(bt, u);
    if (wk.b != X.b) X.load(bt, wk.b, ns, tws, rad);
    if (!X.run) continue;
    const int k = lu / X.upp, ky0 = (lu - k * X.upp) * X.lpw;
    double2 *const S = X.spec + (long long)k * X.nzm * X.nh;
    wfft<SGN, V>(reg, X.N, X.lgL, rad, X.np, tws, WColSrc{S, X.nh, ky0}, WColDst{S, X.nh, ky0});
  }
}

}  // namespace afid
