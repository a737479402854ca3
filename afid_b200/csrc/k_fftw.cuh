// Warp transforms along y (the r2c and c2r steps of
// SolvePressureCorrection.F90:97 and :148) and along z (the c2c steps of
// SolvePressureCorrection.F90:102 and :141).
//
// Each warp transforms LPW = 32 / G complex lines of length N on its own:
// G lanes per line, V = N / G values per lane (8 or 12).  The plan is a mixed-radix
// Stockham sequence whose radices all divide V, so in every pass each lane
// computes exactly V / R butterflies of radix R (no idle lanes).  Passes
// exchange data through a buffer in the warp's own slice of shared memory
// (LPW lines x N values, interleaved n * LPW + line) with __syncwarp only:
// warps never wait for each other.
//
// Warps are independent: a warp unit is LPW lines of one plane of one box
// (2 LPW rows for y, LPW neighbouring ky columns for z), the units of a
// launch are numbered across its boxes, and each warp of the (persistent)
// grid takes runs of consecutive units (4, or 2 or 1 in a launch with
// fewer than 4 units per warp), the runs dealt round-robin over all warps.  A warp keeps the fields of its current box in registers
// and that box's twiddles and radices in its slice, reloading them (with
// __syncwarp only) when its unit belongs to another box: a block has no
// barrier at all.
//
// Each warp pipelines its units through two buffers: while it transforms
// one unit in one buffer, the inputs of its next unit are on their way into
// the other (cp.async, 16 bytes per lane and copy), so the HBM latency of a
// unit's loads overlaps the previous unit's passes.  The outputs leave from
// the last pass (or the unpack) straight to HBM.
#pragma once
#include "k_fft.cuh"

namespace afid {

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

// Warps per block: 8 at V = 8, 6 at V = 12, so that two blocks with their
// double buffers fit an SM's shared memory.
__host__ __device__ constexpr int wf_warps(int V) { return V == 12 ? 6 : 8; }
// One buffer (complex values): the LPW x N values of the passes (32 V), or
// the staged inputs of a unit: 2 LPW padded real rows (2 LPW (N + 2)
// doubles) for the forward y transform, 2 LPW half-spectrum rows (2 LPW
// (N/2 + 1) values) for the inverse; with G >= 2 lanes per line (LPW <= 16)
// both fit in 32 V + 32.
__host__ __device__ constexpr int wf_buf(int V) { return 32 * V + 32; }

// Index of line l's value n in a warp buffer: n LPW + l, plus one complex of
// pad per 8 values of n.  Without the pad, a radix-8 pass writes the eight
// values of each lane's butterfly 8 rows (8 LPW complex) apart, which for
// LPW = 4 is 512 bytes: the same banks for all lanes.  N LPW + N / 8 <= 32 V
// + 16 fits the buffer.
__device__ __forceinline__ int wsidx(int l, int n, int lgL) { return (n << lgL) + l + (n >> 3); }
struct WSmemDst {
  double2 *a;
  int lgL;
  __device__ __forceinline__ void operator()(int l, int n, double2 v) const { a[wsidx(l, n, lgL)] = v; }
};
struct WSmemSrc {
  const double2 *a;
  int lgL;
  __device__ __forceinline__ double2 operator()(int l, int n) const { return a[wsidx(l, n, lgL)]; }
};
// A warp's slice: twiddles (WF_MAX_N complex), radices (8 ints, 32 bytes),
// then the two buffers.
__host__ __device__ constexpr int wf_slice(int V) { return WF_MAX_N + 2 + 2 * wf_buf(V); }
__host__ __device__ constexpr size_t wf_smem_bytes(int V) { return (size_t)wf_warps(V) * wf_slice(V) * 16; }

// The unit sequence of a warp: runs gw, gw + NW, gw + 2 NW, ... of units
// (gw: the warp's index in the grid of W-warp blocks, NW: the grid's warps;
// run lengths as for the tile kernels' TileRange).
template <int W>
struct WarpUnits {
  int gw, nw, total, lgr;
  __device__ __forceinline__ explicit WarpUnits(int total_)
      : gw((int)(blockIdx.x * W + (threadIdx.x >> 5))), nw((int)(gridDim.x * W)), total(total_),
        lgr(run_log2(total_, (int)(gridDim.x * W))) {}
  __device__ __forceinline__ int first() const { return (gw << lgr) < total ? (gw << lgr) : total; }
  __device__ __forceinline__ int next(int u) const {
    int n = u + 1;
    if ((n & ((1 << lgr) - 1)) == 0) n = ((u >> lgr) + nw) << lgr;
    return n < total ? n : total;
  }
};

// The fields of a box a warp transform needs, held in registers.  fields()
// reads the geometry and pointers; load() also reads the box's run state and
// copies its twiddles and radices into the warp's slice.  ZDIR selects the z
// plan: lines of nzm points, LPW columns per unit.
template <bool ZDIR = false>
struct WarpBox {
  int b, N, nzm, nh, lpw, lgL, upp, np;
  long long plane;
  double *phi;
  double2 *spec;
  bool run;
  __device__ __forceinline__ void fields(const BatchDev &bt, int bi) {
    const BoxDev *Bp = bt.boxes + bi;
    b = bi;
    nzm = __ldg(&Bp->nzm);
    nh = __ldg(&Bp->nymh);
    N = ZDIR ? nzm : __ldg(&Bp->nym);
    lpw = 32 / __ldg(ZDIR ? &Bp->wz_g : &Bp->wy_g);
    lgL = ilog2(lpw);
    upp = ZDIR ? (nh + lpw - 1) / lpw : (nzm + 2 * lpw - 1) / (2 * lpw);
    np = __ldg(ZDIR ? &Bp->wz_np : &Bp->wy_np);
    plane = __ldg(&Bp->plane);
    phi = (double *)__ldg((const unsigned long long *)&Bp->phi);
    spec = (double2 *)__ldg((const unsigned long long *)&Bp->spec);
  }
  __device__ __forceinline__ void load(const BatchDev &bt, int bi, int ns, double2 *tws, int *rad) {
    fields(bt, bi);
    const BoxDev *Bp = bt.boxes + bi;
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
  const WSmemSrc as{a, lgL};
  const WSmemDst ad{a, lgL};
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

// first pass of the forward transform: line p = the staged real rows
// (2p, 2p+1) of the unit (row r at rows + r RS doubles; rows beyond the box
// were staged as zeros)
struct WStagedRowPairSrc {
  const double *rows;
  int RS;
  __device__ __forceinline__ double2 operator()(int p, int n) const {
    return make_double2(rows[(2 * p) * RS + n], rows[(2 * p + 1) * RS + n]);
  }
};

// first pass of the inverse transform: line p = the complex line
// A + i B of the staged half-spectrum rows (2p, 2p+1) (rows beyond the box
// are zero), with the Hermitian extension (the imaginary parts at ky = 0 and
// ky = N/2 ignored, as in a c2r transform)
struct WHalfPairSrc {
  const double2 *rows;  // staged row r at rows + r nh
  int N, nh;
  __device__ __forceinline__ double2 coef(int r, int n) const {
    const int q = n < nh ? n : N - n;
    double2 c = rows[r * nh + q];
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
// last pass of the z transform: column ky0 + l of one plane's spectrum (row
// pitch nh), columns at or beyond nh not stored
struct WColDst {
  double2 *S;
  int nh, ky0;
  __device__ __forceinline__ void operator()(int l, int n, double2 v) const {
    if (ky0 + l < nh) __stcg(S + (long long)n * nh + ky0 + l, v);
  }
};

enum { WK_YF = 0, WK_YI = 1, WK_Z = 2 };

// Issue the copies of unit lu's inputs into buffer a (each lane its share,
// cp.async 16 bytes at a time; the entries beyond the box are zeroed).
//   WK_YF: the unit's 2 LPW real rows, contiguous in HBM, to padded rows of
//          RS = N + 2 doubles (the pad spreads the rows of one pass read over
//          the shared-memory banks);
//   WK_YI: the unit's 2 LPW half-spectrum rows, contiguous in HBM;
//   WK_Z:  the unit's LPW columns, kz row by kz row (LPW consecutive values
//          of each row), to a[wsidx(l, n)], the layout of the passes.
template <int KIND, bool ZD>
__device__ __forceinline__ void wf_issue(const WarpBox<ZD> &P, int lu, double2 *a) {
  const int lane = threadIdx.x & 31;
  const double2 zero = make_double2(0.0, 0.0);
  if constexpr (KIND == WK_Z) {
    const int k = lu / P.upp, ky0 = (lu - k * P.upp) * P.lpw;
    const double2 *S = P.spec + (long long)k * P.nzm * P.nh + ky0;
    const int ne = P.N << P.lgL, lmask = P.lpw - 1;
    for (int e = lane; e < ne; e += 32) {
      const int n = e >> P.lgL, l = e & lmask;
      double2 *d = a + wsidx(l, n, P.lgL);
      if (ky0 + l < P.nh) cp_async16(d, S + (long long)n * P.nh + l);
      else *d = zero;
    }
  } else {
    const int k = lu / P.upp, i0 = (lu - k * P.upp) * 2 * P.lpw;
    const int nrow = min(2 * P.lpw, P.nzm - i0);
    if constexpr (KIND == WK_YF) {
      const double *src = P.phi + (long long)k * P.plane + (long long)i0 * P.N;
      const int half = P.N >> 1, RS = P.N + 2, nch = 2 * P.lpw * half;
      double *ad = reinterpret_cast<double *>(a);
      for (int e = lane; e < nch; e += 32) {
        const int r = e / half, c = e - r * half;
        double *d = ad + r * RS + 2 * c;
        if (r < nrow) cp_async16(d, src + (long long)r * P.N + 2 * c);
        else *reinterpret_cast<double2 *>(d) = zero;
      }
    } else {
      const double2 *src = P.spec + (long long)k * P.nzm * P.nh + (long long)i0 * P.nh;
      const int nval = 2 * P.lpw * P.nh, nin = nrow * P.nh;
      for (int e = lane; e < nval; e += 32) {
        if (e < nin) cp_async16(a + e, src + e);
        else a[e] = zero;
      }
    }
  }
}

// Transform unit lu of box X from its staged inputs in buffer a (the passes
// run in place in a) and store its outputs.
template <int KIND, int SGN, int V, bool ZD>
__device__ __forceinline__ void wf_process(const WarpBox<ZD> &X, int lu, double2 *a, const double2 *tws,
                                           const int *rad) {
  const int N = X.N, lpw = X.lpw, lgL = X.lgL, nh = X.nh;
  if constexpr (KIND == WK_Z) {
    const int k = lu / X.upp, ky0 = (lu - k * X.upp) * lpw;
    double2 *const S = X.spec + (long long)k * X.nzm * nh;
    wfft<SGN, V>(a, N, lgL, rad, X.np, tws, WSmemSrc{a, lgL}, WColDst{S, nh, ky0});
  } else {
    const int k = lu / X.upp, i0 = (lu - k * X.upp) * 2 * lpw;
    const int nrow = min(2 * lpw, X.nzm - i0);
    if constexpr (KIND == WK_YF) {
      wfft<-1, V>(a, N, lgL, rad, X.np, tws, WStagedRowPairSrc{reinterpret_cast<const double *>(a), N + 2},
                  WSmemDst{a, lgL});
      // unpack the two real transforms of line l: A = (Z_q + conj Z_{N-q}) / 2,
      // B = (Z_q - conj Z_{N-q}) / (2i), q <= N/2
      const int lane = threadIdx.x & 31;
      const int l = lane & (lpw - 1), g = 32 / lpw;
      double2 *const speck = X.spec + (long long)k * X.nzm * nh;
      const int i = i0 + 2 * l;
      for (int q = lane >> lgL; q < nh; q += g) {
        const double2 z = a[wsidx(l, q, lgL)];
        const double2 zn = a[wsidx(l, q == 0 ? 0 : N - q, lgL)];
        const double2 A = make_double2((z.x + zn.x) * 0.5, (z.y - zn.y) * 0.5);
        const double2 Bv = make_double2((z.y + zn.y) * 0.5, (zn.x - z.x) * 0.5);
        if (i < X.nzm) __stcg(speck + (long long)i * nh + q, A);
        if (i + 1 < X.nzm) __stcg(speck + (long long)(i + 1) * nh + q, Bv);
      }
    } else {
      double *rows = X.phi + (long long)k * X.plane + (long long)i0 * N;
      wfft<+1, V>(a, N, lgL, rad, X.np, tws, WHalfPairSrc{a, N, nh}, WRowPairDst{rows, N, nrow});
    }
  }
}

// The warp's loop over its units, two buffers deep: the copies of unit u+1
// are issued before unit u is transformed.  Each iteration commits one copy
// group (empty after the last unit), so "all groups but the newest done"
// means the current unit's inputs have landed.
template <int KIND, int SGN, int V>
__device__ __forceinline__ void wf_units(const BatchDev &bt, int ns, int total) {
  constexpr bool ZD = (KIND == WK_Z);
  extern __shared__ double2 wsm[];
  double2 *const tws = wsm + (threadIdx.x >> 5) * wf_slice(V);   // this warp's slice
  int *const rad = reinterpret_cast<int *>(tws + WF_MAX_N);
  double2 *const buf0 = tws + WF_MAX_N + 2;
  const WarpUnits<wf_warps(V)> wu(total);
  int u = wu.first();
  if (u >= total) return;
  TileWalk wn(bt, u);
  WarpBox<ZD> X, P;   // boxes of the unit transformed and of the unit copied in
  X.b = -1;
  int lu = wn.to(bt, u), ub = wn.b;
  P.fields(bt, ub);
  wf_issue<KIND>(P, lu, buf0);
  cp_async_commit();
  int cur = 0;
  while (u < total) {
    const int un = wu.next(u);
    int lun = 0, ubn = ub;
    if (un < total) {
      lun = wn.to(bt, un);
      ubn = wn.b;
      if (ubn != P.b) P.fields(bt, ubn);
      wf_issue<KIND>(P, lun, cur ? buf0 : buf0 + wf_buf(V));
    }
    cp_async_commit();
    cp_async_wait_1();
    __syncwarp();
    double2 *const a = cur ? buf0 + wf_buf(V) : buf0;
    if (ub != X.b) X.load(bt, ub, ns, tws, rad);
    if (X.run) wf_process<KIND, SGN, V>(X, lu, a, tws, rad);
    __syncwarp();   // every lane is done with a before the next iteration's copies go into it
    u = un;
    lu = lun;
    ub = ubn;
    cur ^= 1;
  }
  cp_async_wait_all();
}

// Forward (r2c) y transform of the units of the launch.
template <int V>
__global__ void __launch_bounds__(32 * wf_warps(V), 2) k_fftw_y_fwd(BatchDev bt, int ns, int total) {
  wf_units<WK_YF, -1, V>(bt, ns, total);
}

// Inverse (c2r) y transform of the units of the launch.
template <int V>
__global__ void __launch_bounds__(32 * wf_warps(V), 2) k_fftw_y_inv(BatchDev bt, int ns, int total) {
  wf_units<WK_YI, +1, V>(bt, ns, total);
}

// c2c z transform (SGN -1 forward, +1 inverse) of the units of the launch,
// in place in the spectrum: a unit is LPW neighbouring ky columns of one
// plane, so the lanes copying one kz row of the unit read LPW consecutive
// complex values, and the runs of units that neighbouring warps take cover
// neighbouring columns of the rows.
template <int SGN, int V>
__global__ void __launch_bounds__(32 * wf_warps(V), 2) k_fftw_z(BatchDev bt, int ns, int total) {
  wf_units<WK_Z, SGN, V>(bt, ns, total);
}

}  // namespace afid
