// Pressure Poisson solve of SolvePressureCorrection.F90:35-151 on one GPU:
//   y: real-to-complex FFT (two real rows packed in one complex line) of dph;
//   z: complex FFT along kz on tiles of consecutive ky (in place), the tiles
//      brought in by TMA;
//   x: one complex tridiagonal per (ky, kz), Thomas in dgttrf/dgttrs order;
//   then the inverse z and y transforms, the latter writing dph.
// The 2DECOMP pencil transposes of the reference disappear: each transform
// reads its lines directly from the plane-major layout.
//
// The FFTs are Stockham auto-sort passes of radix 16, 8, 4, 2, 3, 5 and 7
// (plans in increasing radix order, e.g. 768 = 3 x 16 x 16), run in place in
// shared memory on tiles copied in with cp.async; the last pass of the z and
// inverse-y transforms streams back to global memory.  Twiddles
// exp(-2 pi i n / N) come from a table computed on the host in extended
// precision and copied to shared memory by every block.
#pragma once
#include "afid_device.cuh"

namespace afid {

// Butterflies of the unnormalised DFT with exponent sign SGN (-1 forward,
// +1 inverse), a compile-time constant so that every multiplication by +-i
// and every conjugation is a sign flip.
template <int SGN>
__device__ __forceinline__ double2 cmul_wi(double2 a, double c, double s) {
  // a * (c + i SGN s)
  const double ss = SGN > 0 ? s : -s;
  return make_double2(a.x * c - a.y * ss, a.x * ss + a.y * c);
}
template <int SGN>
__device__ __forceinline__ double2 mul_sgn_i(double2 a) {   // a * (SGN i)
  return SGN > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}
template <int SGN>
__device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2, double2 &a3) {
  const double2 t0 = cadd(a0, a2), t1 = csub(a0, a2);
  const double2 t2 = cadd(a1, a3), t3 = csub(a1, a3);
  const double2 wt3 = mul_sgn_i<SGN>(t3);
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, wt3);
  a3 = csub(t1, wt3);
}

// three-point DFT in place: X[k] = sum_n a_n W3^(n k), W3 = exp(SGN 2 pi i / 3)
template <int SGN>
__device__ __forceinline__ void dft3(double2 &a0, double2 &a1, double2 &a2) {
  constexpr double S3 = 0.86602540378443864676;   // sin(2 pi / 3)
  const double2 s = cadd(a1, a2), d = csub(a1, a2);
  const double2 m = make_double2(a0.x - 0.5 * s.x, a0.y - 0.5 * s.y);
  const double2 id = make_double2((-SGN * S3) * d.y, (SGN * S3) * d.x);
  a0 = cadd(a0, s);
  a1 = cadd(m, id);
  a2 = csub(m, id);
}

template <int R, int SGN>
__device__ __forceinline__ void dft_small(double2 (&v)[R], const double2 *tw, int N) {
  constexpr double H = 0.70710678118654752440;    // cos(pi/4)
  constexpr double C8 = 0.92387953251128675613;   // cos(pi/8)
  constexpr double S8 = 0.38268343236508977173;   // sin(pi/8)
  if constexpr (R == 2) {
    const double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    dft4<SGN>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    // 8 = 2 x 4: four-point DFTs over n2 of x[n1 + 2 n2], twiddle W8^(n1 k2),
    // two-point DFTs over n1; X[4 k1 + k2]
    double2 a0 = v[0], a1 = v[2], a2 = v[4], a3 = v[6];
    double2 b0 = v[1], b1 = v[3], b2 = v[5], b3 = v[7];
    dft4<SGN>(a0, a1, a2, a3);
    dft4<SGN>(b0, b1, b2, b3);
    b1 = cmul_wi<SGN>(b1, H, H);
    b2 = mul_sgn_i<SGN>(b2);
    b3 = cmul_wi<SGN>(b3, -H, H);
    v[0] = cadd(a0, b0); v[4] = csub(a0, b0);
    v[1] = cadd(a1, b1); v[5] = csub(a1, b1);
    v[2] = cadd(a2, b2); v[6] = csub(a2, b2);
    v[3] = cadd(a3, b3); v[7] = csub(a3, b3);
  } else if constexpr (R == 16) {
    // 16 = 4 x 4: four-point DFTs over n2 of x[n1 + 4 n2] (results Y[n1][k2]
    // kept in v[n1 + 4 k2]), twiddle by W16^(n1 k2), four-point DFTs over n1
    // (X[4 k1 + k2] lands in v[4 k2 + k1]), then a register renaming into
    // natural order.
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) dft4<SGN>(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
    v[5] = cmul_wi<SGN>(v[5], C8, S8);        // n1=1 k2=1: m=1
    v[9] = cmul_wi<SGN>(v[9], H, H);          // n1=1 k2=2: m=2
    v[13] = cmul_wi<SGN>(v[13], S8, C8);      // n1=1 k2=3: m=3
    v[6] = cmul_wi<SGN>(v[6], H, H);          // n1=2 k2=1: m=2
    v[10] = mul_sgn_i<SGN>(v[10]);            // n1=2 k2=2: m=4
    v[14] = cmul_wi<SGN>(v[14], -H, H);       // n1=2 k2=3: m=6
    v[7] = cmul_wi<SGN>(v[7], S8, C8);        // n1=3 k2=1: m=3
    v[11] = cmul_wi<SGN>(v[11], -H, H);       // n1=3 k2=2: m=6
    v[15] = cmul_wi<SGN>(v[15], -C8, -S8);    // n1=3 k2=3: m=9
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) dft4<SGN>(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3]);
    // X[4 k1 + k2] = v[4 k2 + k1]: transpose the 4 x 4 index grid
    double2 t;
    t = v[1]; v[1] = v[4]; v[4] = t;
    t = v[2]; v[2] = v[8]; v[8] = t;
    t = v[3]; v[3] = v[12]; v[12] = t;
    t = v[6]; v[6] = v[9]; v[9] = t;
    t = v[7]; v[7] = v[13]; v[13] = t;
    t = v[11]; v[11] = v[14]; v[14] = t;
  } else if constexpr (R == 3) {
    dft3<SGN>(v[0], v[1], v[2]);
  } else if constexpr (R == 6) {
    // 6 = 2 x 3: three-point DFTs of the even and odd samples, then
    // X[k] = E[k] + W6^k O[k], X[k+3] = E[k] - W6^k O[k]
    constexpr double S3 = 0.86602540378443864676;   // sin(pi / 3)
    double2 e0 = v[0], e1 = v[2], e2 = v[4], o0 = v[1], o1 = v[3], o2 = v[5];
    dft3<SGN>(e0, e1, e2);
    dft3<SGN>(o0, o1, o2);
    o1 = cmul_wi<SGN>(o1, 0.5, S3);     // W6^1
    o2 = cmul_wi<SGN>(o2, -0.5, S3);    // W6^2
    v[0] = cadd(e0, o0); v[3] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[4] = csub(e1, o1);
    v[2] = cadd(e2, o2); v[5] = csub(e2, o2);
  } else if constexpr (R == 12) {
    // 12 = 3 x 4: four-point DFTs over n2 of x[n1 + 3 n2] (Y[n1][k2] kept in
    // slot n1 + 3 k2), twiddle by W12^(n1 k2), three-point DFTs over n1
    // (X[k2 + 4 k1] lands in slot 3 k2 + k1), then a register renaming into
    // natural order
    constexpr double S3 = 0.86602540378443864676;   // sin(pi / 3) = cos(pi / 6)
#pragma unroll
    for (int n1 = 0; n1 < 3; ++n1) dft4<SGN>(v[n1], v[n1 + 3], v[n1 + 6], v[n1 + 9]);
    v[4] = cmul_wi<SGN>(v[4], S3, 0.5);      // n1=1 k2=1: W12^1
    v[7] = cmul_wi<SGN>(v[7], 0.5, S3);      // n1=1 k2=2: W12^2
    v[10] = mul_sgn_i<SGN>(v[10]);           // n1=1 k2=3: W12^3
    v[5] = cmul_wi<SGN>(v[5], 0.5, S3);      // n1=2 k2=1: W12^2
    v[8] = cmul_wi<SGN>(v[8], -0.5, S3);     // n1=2 k2=2: W12^4
    v[11] = make_double2(-v[11].x, -v[11].y);  // n1=2 k2=3: W12^6
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) dft3<SGN>(v[3 * k2], v[3 * k2 + 1], v[3 * k2 + 2]);
    double2 t[12];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2)
#pragma unroll
      for (int k1 = 0; k1 < 3; ++k1) t[k2 + 4 * k1] = v[3 * k2 + k1];
#pragma unroll
    for (int q = 0; q < 12; ++q) v[q] = t[q];
  } else if constexpr (R == 5) {
    const double C1 = 0.30901699437494742410, C2 = -0.80901699437494742410;
    const double S1 = 0.95105651629515357212, S2 = 0.58778525229247312917;
    const double2 a0 = v[0];
    const double2 s14 = cadd(v[1], v[4]), d14 = csub(v[1], v[4]);
    const double2 s23 = cadd(v[2], v[3]), d23 = csub(v[2], v[3]);
    const double2 r1 = make_double2(a0.x + C1 * s14.x + C2 * s23.x, a0.y + C1 * s14.y + C2 * s23.y);
    const double2 r2 = make_double2(a0.x + C2 * s14.x + C1 * s23.x, a0.y + C2 * s14.y + C1 * s23.y);
    const double2 q1 = make_double2(S1 * d14.x + S2 * d23.x, S1 * d14.y + S2 * d23.y);
    const double2 q2 = make_double2(S2 * d14.x - S1 * d23.x, S2 * d14.y - S1 * d23.y);
    const double2 iq1 = mul_sgn_i<SGN>(q1);
    const double2 iq2 = mul_sgn_i<SGN>(q2);
    v[0] = make_double2(a0.x + s14.x + s23.x, a0.y + s14.y + s23.y);
    v[1] = cadd(r1, iq1);
    v[4] = csub(r1, iq1);
    v[2] = cadd(r2, iq2);
    v[3] = csub(r2, iq2);
  } else {
    // generic small radix through the length-N twiddle table (R divides N)
    double2 out[R];
    const int step = N / R;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      double2 acc = v[0];
#pragma unroll
      for (int m = 1; m < R; ++m) {
        double2 w = tw[((m * q) % R) * step];
        if (SGN > 0) w.y = -w.y;
        acc = cadd(acc, cmul(v[m], w));
      }
      out[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = out[q];
  }
}

// Stockham passes over L lines of length N.  Pass p with radix R reads
// element j + r N/R of each butterfly j and writes element
// (j / Ns) Ns R + j % Ns + r Ns, Ns being the product of the earlier radices.
// Passes run in place in one shared buffer: every thread first loads the
// inputs of all its butterflies into registers, the block synchronises, and
// the outputs are stored into the same buffer (then the block synchronises
// again).  A thread takes at most 16 / R butterflies, i.e. holds at most 16
// complex values, so a tile may hold at most FFT_TILE_MAX values.  The first
// pass may read through a source functor (pairs of real rows, raw
// half-spectrum rows) and the last pass may write through a destination
// functor (global memory).  LINE_MAJOR: element (l, n) at l*N + n, else at
// n*L + l.
constexpr int FFT_T = 256;                  // threads per FFT block
constexpr int FFT_TILE_MAX = 14 * FFT_T;    // complex values per tile (radix 7: 2 butterflies of 7)

// Division by a positive int that is usually a power of two (lines per
// tile always are; Ns is for plans with at most one odd radix).
struct FastDiv {
  int d, sh;
  bool p2;
  __device__ __forceinline__ explicit FastDiv(int d_) : d(d_), sh(0), p2((d_ & (d_ - 1)) == 0) {
    while ((2 << sh) <= d) ++sh;
  }
  __device__ __forceinline__ int div(int n) const { return p2 ? (n >> sh) : n / d; }
  __device__ __forceinline__ int mod(int n) const { return p2 ? (n & (d - 1)) : n % d; }
};

template <int R, int SGN>
__device__ __forceinline__ void twiddle(double2 (&v)[R], int k, int tstr, const double2 *tw) {
#pragma unroll
  for (int r = 1; r < R; ++r) {
    double2 w = tw[r * k * tstr];
    if (SGN > 0) w.y = -w.y;
    v[r] = cmul(v[r], w);
  }
}

// element (l, n) of a tile of L lines (L a power of two) at n*L + l
__device__ __forceinline__ int sidx(int l, int n, int lgL) { return (n << lgL) + l; }

template <int R, int SGN, class Src, class Dst>
__device__ __forceinline__ void pass_inplace(int N, int lgL, int Ns, const double2 *tw,
                                             const Src &src, const Dst &dst) {
  constexpr int BPT = 16 / R;               // butterflies per thread
  const int NR = N / R, tstr = N / (Ns * R);
  const int lmask = (1 << lgL) - 1;
  const FastDiv dNs(Ns);
  double2 v[BPT][R];
  // thread t takes butterflies j = t / L + b FFT_T / L of line l = t % L;
  // idle slots hold zeros (v must be defined on every path to stay in
  // registers across the barrier)
  const int l = threadIdx.x & lmask, j0 = threadIdx.x >> lgL, jstep = FFT_T >> lgL;
#pragma unroll
  for (int b = 0; b < BPT; ++b) {
    const int j = j0 + b * jstep;
#pragma unroll
    for (int r = 0; r < R; ++r) v[b][r] = make_double2(0.0, 0.0);
    if (j < NR) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = src(l, j + r * NR);
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < BPT; ++b) {
    const int j = j0 + b * jstep;
    if (j < NR) {
      const int k = dNs.mod(j);
      if (Ns > 1) twiddle<R, SGN>(v[b], k, tstr, tw);
      dft_small<R, SGN>(v[b], tw, N);
      const int base = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) dst(l, base + r * Ns, v[b][r]);
    }
  }
  __syncthreads();
}

template <int SGN, class Src, class Dst>
__device__ __forceinline__ void run_inplace(int R, int N, int lgL, int Ns, const double2 *tw,
                                            const Src &src, const Dst &dst) {
  switch (R) {
    case 16: pass_inplace<16, SGN>(N, lgL, Ns, tw, src, dst); break;
    case 8: pass_inplace<8, SGN>(N, lgL, Ns, tw, src, dst); break;
    case 4: pass_inplace<4, SGN>(N, lgL, Ns, tw, src, dst); break;
    case 2: pass_inplace<2, SGN>(N, lgL, Ns, tw, src, dst); break;
    case 3: pass_inplace<3, SGN>(N, lgL, Ns, tw, src, dst); break;
    case 5: pass_inplace<5, SGN>(N, lgL, Ns, tw, src, dst); break;
    default: pass_inplace<7, SGN>(N, lgL, Ns, tw, src, dst); break;
  }
}

struct SmemDst {
  double2 *a; int lgL;
  __device__ __forceinline__ void operator()(int l, int n, double2 v) const { a[sidx(l, n, lgL)] = v; }
};
struct SmemSrc {
  const double2 *a; int lgL;
  __device__ __forceinline__ double2 operator()(int l, int n) const { return a[sidx(l, n, lgL)]; }
};

// Whole transform of a tile held in shared buffer a: the first pass reads
// ``src``, the last pass writes ``dst`` when LAST_TO_DST (otherwise the
// result stays in a).
template <bool LAST_TO_DST, int SGN, class Src, class Dst>
__device__ void fft_tile(double2 *a, int N, int lgL, const int *rad, int np, const double2 *tw,
                         const Src &src, const Dst &dst) {
  const SmemSrc as{a, lgL};
  const SmemDst ad{a, lgL};
  if (np == 1) {
    if (LAST_TO_DST) run_inplace<SGN>(rad[0], N, lgL, 1, tw, src, dst);
    else run_inplace<SGN>(rad[0], N, lgL, 1, tw, src, ad);
    return;
  }
  run_inplace<SGN>(rad[0], N, lgL, 1, tw, src, ad);
  int Ns = rad[0];
  for (int p = 1; p < np - 1; ++p) {
    run_inplace<SGN>(rad[p], N, lgL, Ns, tw, as, ad);
    Ns *= rad[p];
  }
  if (LAST_TO_DST) run_inplace<SGN>(rad[np - 1], N, lgL, Ns, tw, as, dst);
  else run_inplace<SGN>(rad[np - 1], N, lgL, Ns, tw, as, ad);
}

// Persistent transform blocks.  A launch has at most (SMs x resident blocks)
// blocks; each takes runs of tiles (TileRange) and copies the next tile into
// its second shared-memory slot (bulk copy or TMA) while it transforms the
// current one in place.  Shared memory: two slots and the
// twiddles of the box being transformed.  Lines per tile default to what
// keeps two blocks on an SM (and at most FFT_TILE_MAX values per tile); the
// tuning fields may choose other values within those limits.
constexpr int FFT_SMEM_DEFAULT = 110 * 1024;
constexpr int FFT_SMEM_MAX = 200 * 1024;
constexpr int FFT_MAX_LINES = 64;      // lines per tile the tuning may ask for
constexpr int FFT_DEFAULT_LINES = 16;  // and the built-in choice at most

// y: a slot holds the 2 Pp real rows of a forward tile (Pp N complex) or the
// 2 Pp half-spectrum rows of an inverse tile (2 Pp (N/2+1) complex)
__host__ __device__ __forceinline__ int fft_y_slot(int N, int Pp) { return 2 * Pp * (N / 2 + 1); }  // = Pp (N + 2)
// Dynamic shared memory of a transform block: two slots, the twiddles, then
// the two slot mbarriers (16 bytes) and the cached box descriptor.  The
// slots come first, at the start of the dynamic region, which keeps the TMA
// destinations aligned (the block has no static shared memory).
constexpr int FFT_DESC_BYTES = (int)((sizeof(BoxDev) + 15) / 16 * 16);
constexpr int FFT_TAIL_BYTES = 16 + FFT_DESC_BYTES;
static_assert(FFT_TAIL_BYTES <= 1024, "the autotuner's size bound assumes a tail of at most 1 KB");
__host__ __device__ __forceinline__ int fft_y_bytes(int N, int Pp) { return (2 * fft_y_slot(N, Pp) + N) * 16 + FFT_TAIL_BYTES; }
__host__ __device__ __forceinline__ int fft_z_bytes(int N, int L) { return (2 * L * N + N) * 16 + FFT_TAIL_BYTES; }
__host__ __device__ __forceinline__ bool fft_pow2(int v) { return v >= 1 && (v & (v - 1)) == 0; }
__host__ __device__ __forceinline__ bool fft_y_ok(int N, int Pp, int budget) {
  return fft_pow2(Pp) && Pp <= FFT_MAX_LINES && Pp * N <= FFT_TILE_MAX && fft_y_bytes(N, Pp) <= budget;
}
__host__ __device__ __forceinline__ bool fft_z_ok(int N, int L, int budget) {
  return fft_pow2(L) && L <= FFT_MAX_LINES && L * N <= FFT_TILE_MAX && fft_z_bytes(N, L) <= budget;
}
__host__ __device__ __forceinline__ int fft_fit_lines(int N, int budget, bool y) {
  int l = FFT_DEFAULT_LINES;
  while (l > 1 && !(y ? fft_y_ok(N, l, budget) : fft_z_ok(N, l, budget))) l >>= 1;
  return l;
}
__host__ __device__ __forceinline__ int ilog2(int v) {
  int r = 0;
  while ((1 << (r + 1)) <= v) ++r;
  return r;
}
__host__ __device__ __forceinline__ int fft_y_pairs(const BoxDev &B) {
  if (B.fy_lines > 0) return B.fy_lines;
  int l = fft_fit_lines(B.nym, FFT_SMEM_DEFAULT, true);
  while (l > 1 && l >= B.nzm) l >>= 1;        // no tile taller than needed
  return l;
}
__host__ __device__ __forceinline__ int fft_z_lines(const BoxDev &B) {
  int l = B.fz_lines > 0 ? B.fz_lines : fft_fit_lines(B.nzm, FFT_SMEM_DEFAULT, false);
  while (l > 1 && l / 2 >= B.nymh) l >>= 1;   // no tile wider than needed
  return l;
}

// shared-memory layout of one launch (largest box of the batch)
struct FftSmem {
  int slot;   // complex values per copy-in slot (the twiddles follow the two slots)
  int tw;     // complex values of the twiddle table (the z transform's mbarriers follow it)
};

// A persistent block takes runs of consecutive tiles, the runs dealt
// round-robin over the blocks (block p: runs p, p + G, p + 2G, ...):
// neighbouring blocks work on neighbouring tiles at the same time, the work
// of boxes of different sizes spreads over all blocks, and a block changes
// boxes at most once per run.  Runs are FFT_TILE_RUN long when every worker
// of the grid (block, or warp of the warp transforms) gets at least that many
// items, else 2 or 1 long, so that a small launch spreads over all workers.
// A walker follows the tiles' boxes forward.
constexpr int FFT_TILE_RUN = 4;
__device__ __forceinline__ int run_log2(int total, int workers) {
  return total >= FFT_TILE_RUN * workers ? 2 : total >= 2 * workers ? 1 : 0;
}
struct TileRange {
  int t0, total, lgr;
  __device__ __forceinline__ explicit TileRange(int total_)
      : total(total_), lgr(run_log2(total_, (int)gridDim.x)) { t0 = (int)blockIdx.x << lgr; }
  __device__ __forceinline__ int first() const { return t0 < total ? t0 : total; }
  __device__ __forceinline__ int next(int t) const {
    int n = t + 1;
    if ((n & ((1 << lgr) - 1)) == 0) n = ((t >> lgr) + (int)gridDim.x) << lgr;
    return n < total ? n : total;
  }
};
struct TileWalk {
  int b, lo, hi;   // box b holds the tiles [lo, hi) of the launch
  __device__ __forceinline__ TileWalk(const BatchDev &bt, int t) {
    b = find_box(bt.tile_off, bt.nbox, t);
    lo = __ldg(bt.tile_off + b);
    hi = __ldg(bt.tile_off + b + 1);
  }
  // advance to the box of tile t >= the current tile; returns t's index in its box
  __device__ __forceinline__ int to(const BatchDev &bt, int t) {
    while (t >= hi) {
      ++b;
      lo = hi;
      hi = __ldg(bt.tile_off + b + 1);
    }
    return t - lo;
  }
};

// A transform block keeps the descriptor of the box it is working on in
// shared memory, next to that box's twiddles, and reloads both when a tile
// of another box comes up.  Read from global memory, every descriptor field
// after a global store would be reloaded (the store might alias it), and
// each reload is a dependent trip to the L2.  The block's threads copy the
// descriptor word by word; the caller synchronises before and after.
__device__ __forceinline__ void fft_load_box(const BatchDev &bt, int b, BoxDev &sb) {
  static_assert(sizeof(BoxDev) % 8 == 0, "BoxDev is copied in 8-byte words");
  for (int w = threadIdx.x; w < (int)(sizeof(BoxDev) / 8); w += FFT_T)
    reinterpret_cast<unsigned long long *>(&sb)[w] =
        __ldg(reinterpret_cast<const unsigned long long *>(bt.boxes + b) + w);
}

// ---------------------------------------------------------------------------
// y forward: rows (k, i) of length nym of dph -> spec[k][i][ky], ky <= nym/2.
// A tile is 2 Pp consecutive rows of one plane; line p of the transform is
// the complex pair (row 2p, row 2p+1), unpacked after the last pass into the
// two half spectra.
// ---------------------------------------------------------------------------
struct NoDst {
  __device__ __forceinline__ void operator()(int, int, double2) const {}
};
// rows are copied in with a stride of nym + 2 doubles, which spreads the
// rows of one column over the shared-memory banks and keeps every row
// 16-byte aligned
struct PairSrc {
  const double *rows; int RS;
  __device__ __forceinline__ double2 operator()(int p, int n) const {
    return make_double2(rows[2 * p * RS + n], rows[(2 * p + 1) * RS + n]);
  }
};

// Copy-in of a y tile: one bulk copy per row (issued by one thread,
// completed on the slot's mbarrier); rows beyond nzm are zeroed by the block.
__device__ __forceinline__ void fft_y_fwd_issue(const BoxDev &B, int lt, double *rows, unsigned long long *bar) {
  const int N = B.nym, nzm = B.nzm, Pp = fft_y_pairs(B);
  const int groups = (nzm + 2 * Pp - 1) / (2 * Pp);
  const int k = lt / groups, i0 = (lt - k * groups) * 2 * Pp;
  const int nr = min(2 * Pp, nzm - i0);
  mbar_expect_tx(bar, (unsigned)(nr * N * 8));
  const double *phik = B.phi + (long long)k * B.plane;
  for (int r = 0; r < nr; ++r) bulk_load(rows + r * (N + 2), phik + (long long)(i0 + r) * N, (unsigned)(N * 8), bar);
}
__device__ __forceinline__ void fft_y_fwd_zero_tail(const BoxDev &B, int lt, double *rows) {
  const int N = B.nym, nzm = B.nzm, Pp = fft_y_pairs(B);
  const int groups = (nzm + 2 * Pp - 1) / (2 * Pp);
  const int i0 = (lt - (lt / groups) * groups) * 2 * Pp;
  for (int r = max(nzm - i0, 0); r < 2 * Pp; ++r)
    for (int j = threadIdx.x; j < N; j += FFT_T) rows[r * (N + 2) + j] = 0.0;
}

__global__ void __launch_bounds__(FFT_T, 2) k_fft_y_fwd(BatchDev bt, int ns, FftSmem sm, int total) {
  extern __shared__ double2 fsm[];
  double2 *slot[2] = {fsm, fsm + sm.slot};
  double2 *tws = fsm + 2 * sm.slot;
  unsigned long long *bar = (unsigned long long *)(tws + sm.tw);
  BoxDev &sb = *reinterpret_cast<BoxDev *>(bar + 2);   // descriptor of the box of the current tile
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const TileRange rg(total);
  if (rg.first() >= total) return;
  TileWalk wk(bt, rg.first()), wn = wk;
  int loaded = -1, lt;
  bool run = false;
  {
    const int l0 = wn.to(bt, rg.first());
    if (threadIdx.x == 0) fft_y_fwd_issue(bt.boxes[wn.b], l0, (double *)slot[0], &bar[0]);
    fft_y_fwd_zero_tail(bt.boxes[wn.b], l0, (double *)slot[0]);
  }
  for (int it = 0, t = rg.first(); t < total; ++it, t = rg.next(t)) {
    const int tn = rg.next(t);
    if (tn < total) {
      const int ln = wn.to(bt, tn);
      const BoxDev &Bn = wn.b == loaded ? sb : bt.boxes[wn.b];
      if (threadIdx.x == 0) fft_y_fwd_issue(Bn, ln, (double *)slot[(it + 1) & 1], &bar[(it + 1) & 1]);
      fft_y_fwd_zero_tail(Bn, ln, (double *)slot[(it + 1) & 1]);
    }
    lt = wk.to(bt, t);
    if (wk.b != loaded) {
      __syncthreads();
      fft_load_box(bt, wk.b, sb);
      __syncthreads();
      for (int q = threadIdx.x; q < sb.nym; q += FFT_T) tws[q] = __ldg(sb.twy + q);
      loaded = wk.b;
      // the box's state, read once per box and made uniform over the block
      run = __syncthreads_and(sb.active && ns < sb.nsst && *(volatile int *)&sb.sc->status == 0);
    }
    const BoxDev &B = sb;
    const bool ok = mbar_wait_bounded(&bar[it & 1], (it >> 1) & 1);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicExch(&B.sc->status, AFID_STATUS_DEVICE_TIMEOUT);
        if (tn < total) mbar_wait_bounded(&bar[(it + 1) & 1], ((it + 1) >> 1) & 1);
      }
      return;
    }
    if (run) {
      const int N = B.nym, nzm = B.nzm, Pp = fft_y_pairs(B), nh = B.nymh;
      const int groups = (nzm + 2 * Pp - 1) / (2 * Pp);
      const int k = lt / groups, i0 = (lt - k * groups) * 2 * Pp;
      double2 *cur = slot[it & 1];
      const int lgP = ilog2(Pp);
      fft_tile<false, -1>(cur, N, lgP, B.fft_y_radix, B.fft_y_np, tws, PairSrc{(const double *)cur, N + 2},
                          NoDst{});
      // unpack the two real transforms: A = (Z_q + conj Z_{N-q}) / 2,
      // B = (Z_q - conj Z_{N-q}) / (2i)
      double2 *const speck = B.spec + (long long)k * nzm * nh;
      for (int u = threadIdx.x; u < Pp * nh; u += FFT_T) {
        const int p = u & (Pp - 1), q = u >> lgP;
        const int i = i0 + 2 * p;
        if (i >= nzm) continue;
        const double2 z = cur[sidx(p, q, lgP)];
        const double2 zn = cur[sidx(p, q == 0 ? 0 : N - q, lgP)];
        const double2 A = make_double2((z.x + zn.x) * 0.5, (z.y - zn.y) * 0.5);
        const double2 Bv = make_double2((z.y + zn.y) * 0.5, (zn.x - z.x) * 0.5);
        const long long base = (long long)i * nh + q;
        __stcg(speck + base, A);
        if (i + 1 < nzm) __stcg(speck + base + nh, Bv);
      }
    }
    // the slot is refilled by bulk copies in the next iteration
    fence_proxy_async_smem();
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// z transform in place on spec[k][kz][ky] for a tile of L consecutive ky.
// The division of the forward transform by nym*nzm
// (SolvePressureCorrection.F90:105) is done by k_poisson_x as it reads each
// value, in the same operation order.
// ---------------------------------------------------------------------------
struct ZDst {
  double2 *spec; int nh, ky0;
  __device__ __forceinline__ void operator()(int l, int n, double2 v) const {
    const int ky = ky0 + l;
    if (ky >= nh) return;
    __stcg(spec + (long long)n * nh + ky, v);
  }
};

// The tile of L consecutive ky at all kz of plane k is a dense box of spec
// seen as a 2-D FP64 array (2 nymh doubles per kz row, nxm nzm rows): one
// thread loads it with nzm / fz_rb TMA copies of 2L x fz_rb doubles, which
// land in shared memory as element (l, kz) at kz L + l; ky beyond nymh reads
// as zero.  The copy of the next tile runs while the current one is
// transformed; each slot completes on its own mbarrier.
__device__ __forceinline__ void fft_z_issue(const BoxDev &B, int lt, double2 *a, unsigned long long *bar) {
  const int N = B.nzm, nh = B.nymh, L = fft_z_lines(B), rb = B.fz_rb;
  const int ntl = (nh + L - 1) / L;
  const int k = lt / ntl, ky0 = (lt - k * ntl) * L;
  mbar_expect_tx(bar, (unsigned)(16 * L * N));
  if (B.z_copy_skip) return;   // test switch: the wait on this slot runs out
  for (int c = 0; c < N / rb; ++c) tma_load_2d(a + c * rb * L, B.tm_z, bar, 2 * ky0, k * N + c * rb);
}

template <int SGN>
__global__ void __launch_bounds__(FFT_T, 2) k_fft_z(BatchDev bt, int ns, FftSmem sm, int total) {
  extern __shared__ double2 fsm[];
  double2 *slot[2] = {fsm, fsm + sm.slot};
  double2 *tws = fsm + 2 * sm.slot;
  unsigned long long *bar = (unsigned long long *)(tws + sm.tw);
  BoxDev &sb = *reinterpret_cast<BoxDev *>(bar + 2);   // descriptor of the box of the current tile
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const TileRange rg(total);
  if (rg.first() >= total) return;
  TileWalk wk(bt, rg.first()), wn = wk;
  int loaded = -1, lt;
  bool run = false;
  {
    const int l0 = wn.to(bt, rg.first());
    if (threadIdx.x == 0) fft_z_issue(bt.boxes[wn.b], l0, slot[0], &bar[0]);
  }
  for (int it = 0, t = rg.first(); t < total; ++it, t = rg.next(t)) {
    const int tn = rg.next(t);
    if (tn < total) {
      const int ln = wn.to(bt, tn);
      if (threadIdx.x == 0)
        fft_z_issue(wn.b == loaded ? sb : bt.boxes[wn.b], ln, slot[(it + 1) & 1], &bar[(it + 1) & 1]);
    }
    lt = wk.to(bt, t);
    if (wk.b != loaded) {
      __syncthreads();
      fft_load_box(bt, wk.b, sb);
      __syncthreads();
      for (int q = threadIdx.x; q < sb.nzm; q += FFT_T) tws[q] = __ldg(sb.twz + q);
      loaded = wk.b;
      run = __syncthreads_and(sb.active && ns < sb.nsst && *(volatile int *)&sb.sc->status == 0);
    }
    const BoxDev &B = sb;
    const unsigned tries = B.mbar_tries ? B.mbar_tries : MBAR_MAX_TRIES;
    const bool ok = mbar_wait_bounded(&bar[it & 1], (it >> 1) & 1, tries);
    if (__syncthreads_or(!ok)) {
      // a copy did not complete: flag the box, let the other slot's copy
      // (if any) finish within the same bound, and stop this block
      if (threadIdx.x == 0) {
        atomicExch(&B.sc->status, AFID_STATUS_DEVICE_TIMEOUT);
        if (tn < total) mbar_wait_bounded(&bar[(it + 1) & 1], ((it + 1) >> 1) & 1, tries);
      }
      return;
    }
    if (run) {
      const int N = B.nzm, nh = B.nymh, L = fft_z_lines(B);
      const int ntl = (nh + L - 1) / L;
      const int k = lt / ntl, ky0 = (lt - k * ntl) * L;
      double2 *cur = slot[it & 1];
      const int lgL = ilog2(L);
      fft_tile<true, SGN>(cur, N, lgL, B.fft_z_radix, B.fft_z_np, tws, SmemSrc{cur, lgL},
                          ZDst{B.spec + (long long)k * N * nh, nh, ky0});
    }
    // the slot is refilled by TMA in the next iteration
    fence_proxy_async_smem();
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// x: complex tridiagonal per mode (SolvePressureCorrection.F90:117-137),
// marching k.  Row k of the normalised system is
//   amph(k) x(k-1) + x(k) + apph(k) x(k+1) = dphc(k) s(k),
//   s(k) = 1 / (acphk(k) - ak2(ky) - ak1(kz)).
// dphc arrives unnormalised from the forward z transform and is scaled by
// 1/(nym*nzm) here, before the scaling by s(k).  Its coefficients are real,
// so the complex Thomas sweep is a real sweep applied to both parts.  The
// (0,0) mode is singular (Neumann in x): its last equation is dropped and its
// last unknown set to zero.
//
// The modified wavenumber is even, ak1(kz) = ak1(nzm - kz) bit for bit
// (InitPressureSolver.F90:28-37 computes both from |kz|), so the modes kz and
// nzm - kz of one ky have the same s(k) and the same pivots: one thread
// solves both, the pivot table holds kz <= nzm/2 only, and the two chains
// of the thread overlap each other's latency.
// ---------------------------------------------------------------------------
constexpr int KP_U = 4;   // planes per prefetch chunk of the sweeps

// Row scale s(k) of mode (ak, ak1) and one step of the pivot recurrence
// (zgttrf without pivoting): for row k >= 1 with am = amph(k) s(k),
//   fact = am / d(k-1),  d(k) = 1 - fact * ap(k-1),  ap(k-1) = apph(k-1) s(k-1).
// The sweep and the kernel that tabulates the pivots both go through these,
// so the table holds the bits the sweep would compute.
__device__ __forceinline__ double px_scale(const double *acph, int k, double ak, double ak1) {
  return 1.0 / ((__ldg(acph + k) - ak) - ak1);
}
__device__ __forceinline__ double px_pivot(double am, double ap_prev, double &d) {
  const double fact = am / d;
  d = 1.0 - fact * ap_prev;
  return fact;
}

// number of (kz <= nzm/2, ky) mode pairs of a box
__host__ __device__ __forceinline__ long long px_pairs(int nzm, int nymh) { return (long long)(nzm / 2 + 1) * nymh; }

// Reciprocal pivots 1/d(k) of the modes kz <= nzm/2 of one box, written to
// B.dstore as [k][kz][ky].  They depend on the grid only, so a box computes
// them once.
__global__ void __launch_bounds__(256) k_poisson_pivots(BoxDev B) {
  const int nh = B.nymh, nzm = B.nzm, nxm = B.nxm;
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long np = px_pairs(nzm, nh);
  if (m >= np) return;
  const int kz = (int)(m / nh), ky = (int)(m - (long long)kz * nh);
  const double ak = __ldg(B.tab + (long long)T_NK * B.nx + nzm + ky);
  const double ak1 = __ldg(B.tab + (long long)T_NK * B.nx + kz);
  const double *amph = B.tab + (long long)T_AMPHK * B.nx;
  const double *acph = B.tab + (long long)T_ACPHK * B.nx;
  const double *apph = B.tab + (long long)T_APPHK * B.nx;
  double *__restrict__ dst = B.dstore + m;
  double d = 1.0, ap_prev = 0.0;
  for (int k = 0; k < nxm; ++k) {
    const double s = px_scale(acph, k, ak, ak1);
    if (k > 0) px_pivot(__ldg(amph + k) * s, ap_prev, d);
    dst[(long long)k * np] = 1.0 / d;
    ap_prev = __ldg(apph + k) * s;
  }
}

// One thread per mode pair (kz, ky), (nzm - kz, ky) with kz <= nzm/2 (the
// pair is a single mode for kz = 0 and kz = nzm/2), marching k: the forward
// vector is written over the spectrum and read back by the back
// substitution.
__global__ void __launch_bounds__(256, 2) k_poisson_x(BatchDev bt, int ns) {
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  if (B.sc->status != 0) return;
  const int nh = B.nymh, nzm = B.nzm, nxm = B.nxm;
  const long long m = (long long)(blockIdx.x - __ldg(bt.tile_off + b)) * blockDim.x + threadIdx.x;
  const long long np = px_pairs(nzm, nh);
  if (m >= np) return;
  const int kz = (int)(m / nh), ky = (int)(m - (long long)kz * nh);
  const bool pair = kz > 0 && 2 * kz != nzm;
  const double ak = __ldg(B.tab + (long long)T_NK * B.nx + nzm + ky);   // ak2(ky)
  const double ak1 = __ldg(B.tab + (long long)T_NK * B.nx + kz);      // ak1(kz) = ak1(nzm - kz)
  const double *amph = B.tab + (long long)T_AMPHK * B.nx;
  const double *acph = B.tab + (long long)T_ACPHK * B.nx;
  const double *apph = B.tab + (long long)T_APPHK * B.nx;
  const long long st = (long long)nzm * nh;                           // plane stride of the spectrum
  double2 *__restrict__ xa = B.spec + (long long)kz * nh + ky;        // mode kz
  double2 *__restrict__ xb = B.spec + (long long)(pair ? nzm - kz : kz) * nh + ky;   // mode nzm - kz
  const double *__restrict__ rdt = B.dstore + m;                      // 1/d(k), by k_poisson_pivots
  const bool zero_mode = (ky == 0 && kz == 0);
  const double inv_norm = 1.0 / ((double)B.nzm * (double)B.nym);     // the transforms' 1/(nym nzm)
  // forward elimination (dgttrf + dgttrs forward sweep), planes in chunks
  double d = 1.0, ap_prev = 0.0;
  double2 ya = make_double2(0.0, 0.0), yb = ya;
  for (int k0 = 0; k0 < nxm; k0 += KP_U) {
    double2 ra[KP_U], rb[KP_U];
#pragma unroll
    for (int u = 0; u < KP_U; ++u)
      if (k0 + u < nxm) {
        ra[u] = xa[(long long)(k0 + u) * st];
        rb[u] = xb[(long long)(k0 + u) * st];   // = ra[u] for a single mode (not stored)
      }
#pragma unroll
    for (int u = 0; u < KP_U; ++u) {
      const int k = k0 + u;
      if (k >= nxm) break;
      const double s = px_scale(acph, k, ak, ak1);
      double2 fa = ra[u], fb = rb[u];
      fa.x = (fa.x * inv_norm) * s; fa.y = (fa.y * inv_norm) * s;
      fb.x = (fb.x * inv_norm) * s; fb.y = (fb.y * inv_norm) * s;
      if (k == 0) {
        ya = fa;
        yb = fb;
      } else {
        const double fact = px_pivot(__ldg(amph + k) * s, ap_prev, d);
        ya.x = fa.x - fact * ya.x; ya.y = fa.y - fact * ya.y;
        yb.x = fb.x - fact * yb.x; yb.y = fb.y - fact * yb.y;
      }
      xa[(long long)k * st] = ya;
      if (pair) xb[(long long)k * st] = yb;
      ap_prev = __ldg(apph + k) * s;
    }
  }
  // back substitution
  double2 xna, xnb;
  {
    const double rd = rdt[(long long)(nxm - 1) * np];
    xna = zero_mode ? make_double2(0.0, 0.0) : make_double2(ya.x * rd, ya.y * rd);
    xnb = make_double2(yb.x * rd, yb.y * rd);
  }
  xa[(long long)(nxm - 1) * st] = xna;
  if (pair) xb[(long long)(nxm - 1) * st] = xnb;
  for (int k0 = nxm - 2; k0 >= 0; k0 -= KP_U) {
    double2 yka[KP_U], ykb[KP_U];
    double rk[KP_U];
#pragma unroll
    for (int u = 0; u < KP_U; ++u) {
      const int k = k0 - u;
      if (k >= 0) {
        yka[u] = xa[(long long)k * st];
        ykb[u] = xb[(long long)k * st];
        rk[u] = rdt[(long long)k * np];
      }
    }
#pragma unroll
    for (int u = 0; u < KP_U; ++u) {
      const int k = k0 - u;
      if (k < 0) break;
      const double sk = px_scale(acph, k, ak, ak1);
      const double ap = __ldg(apph + k) * sk;
      xna.x = (yka[u].x - ap * xna.x) * rk[u];
      xna.y = (yka[u].y - ap * xna.y) * rk[u];
      xnb.x = (ykb[u].x - ap * xnb.x) * rk[u];
      xnb.y = (ykb[u].y - ap * xnb.y) * rk[u];
      xa[(long long)k * st] = xna;
      if (pair) xb[(long long)k * st] = xnb;
    }
  }
}

struct YInvSmemSrc {
  const double2 *raw; int N, nh; bool even;    // raw: [row][nh] for the block's 2*Pp rows
  __device__ __forceinline__ double2 coef(int r, int n) const {
    const int q = n < nh ? n : N - n;
    double2 c = raw[r * nh + q];
    if (q == 0 || (even && 2 * q == N)) c.y = 0.0;
    else if (n >= nh) c.y = -c.y;
    return c;
  }
  __device__ __forceinline__ double2 operator()(int p, int n) const {
    const double2 A = coef(2 * p, n), Bv = coef(2 * p + 1, n);
    return make_double2(A.x - Bv.y, A.y + Bv.x);
  }
};
struct YInvDst {
  double *phi; int N, nzm, i0;
  __device__ __forceinline__ void operator()(int p, int j, double2 v) const {
    const int i = i0 + 2 * p;
    if (i < nzm) __stcg(phi + (long long)i * N + j, v.x);
    if (i + 1 < nzm) __stcg(phi + (long long)(i + 1) * N + j, v.y);
  }
};

// y inverse (complex-to-real, unnormalised): spec[k][i][ky] -> phi[k][i][j].
// As in a c2r transform, the imaginary parts of the ky = 0 and ky = nym/2
// coefficients are ignored.  A tile's 2 Pp half-spectrum rows are copied
// into a slot; two rows are recovered from one complex line Z = A + i B,
// which the first pass writes over the raw rows it has read.
// Copy-in of an inverse y tile: one bulk copy per half-spectrum row (issued
// by one thread, completed on the slot's mbarrier); rows beyond nzm are
// zeroed by the block.
__device__ __forceinline__ void fft_y_inv_issue(const BoxDev &B, int lt, double2 *raw, unsigned long long *bar) {
  const int nzm = B.nzm, nh = B.nymh, Pp = fft_y_pairs(B);
  const int groups = (nzm + 2 * Pp - 1) / (2 * Pp);
  const int k = lt / groups, i0 = (lt - k * groups) * 2 * Pp;
  const int nr = min(2 * Pp, nzm - i0);
  mbar_expect_tx(bar, (unsigned)(nr * nh * 16));
  const double2 *speck = B.spec + (long long)k * nzm * nh;
  for (int r = 0; r < nr; ++r) bulk_load(raw + r * nh, speck + (long long)(i0 + r) * nh, (unsigned)(nh * 16), bar);
}
__device__ __forceinline__ void fft_y_inv_zero_tail(const BoxDev &B, int lt, double2 *raw) {
  const int nzm = B.nzm, nh = B.nymh, Pp = fft_y_pairs(B);
  const int groups = (nzm + 2 * Pp - 1) / (2 * Pp);
  const int i0 = (lt - (lt / groups) * groups) * 2 * Pp;
  for (int r = max(nzm - i0, 0); r < 2 * Pp; ++r)
    for (int q = threadIdx.x; q < nh; q += FFT_T) raw[r * nh + q] = make_double2(0.0, 0.0);
}

__global__ void __launch_bounds__(FFT_T, 2) k_fft_y_inv(BatchDev bt, int ns, FftSmem sm, int total) {
  extern __shared__ double2 fsm[];
  double2 *slot[2] = {fsm, fsm + sm.slot};
  double2 *tws = fsm + 2 * sm.slot;
  unsigned long long *bar = (unsigned long long *)(tws + sm.tw);
  BoxDev &sb = *reinterpret_cast<BoxDev *>(bar + 2);   // descriptor of the box of the current tile
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const TileRange rg(total);
  if (rg.first() >= total) return;
  TileWalk wk(bt, rg.first()), wn = wk;
  int loaded = -1, lt;
  bool run = false;
  {
    const int l0 = wn.to(bt, rg.first());
    if (threadIdx.x == 0) fft_y_inv_issue(bt.boxes[wn.b], l0, slot[0], &bar[0]);
    fft_y_inv_zero_tail(bt.boxes[wn.b], l0, slot[0]);
  }
  for (int it = 0, t = rg.first(); t < total; ++it, t = rg.next(t)) {
    const int tn = rg.next(t);
    if (tn < total) {
      const int ln = wn.to(bt, tn);
      const BoxDev &Bn = wn.b == loaded ? sb : bt.boxes[wn.b];
      if (threadIdx.x == 0) fft_y_inv_issue(Bn, ln, slot[(it + 1) & 1], &bar[(it + 1) & 1]);
      fft_y_inv_zero_tail(Bn, ln, slot[(it + 1) & 1]);
    }
    lt = wk.to(bt, t);
    if (wk.b != loaded) {
      __syncthreads();
      fft_load_box(bt, wk.b, sb);
      __syncthreads();
      for (int q = threadIdx.x; q < sb.nym; q += FFT_T) tws[q] = __ldg(sb.twy + q);
      loaded = wk.b;
      run = __syncthreads_and(sb.active && ns < sb.nsst && *(volatile int *)&sb.sc->status == 0);
    }
    const BoxDev &B = sb;
    const bool ok = mbar_wait_bounded(&bar[it & 1], (it >> 1) & 1);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicExch(&B.sc->status, AFID_STATUS_DEVICE_TIMEOUT);
        if (tn < total) mbar_wait_bounded(&bar[(it + 1) & 1], ((it + 1) >> 1) & 1);
      }
      return;
    }
    if (run) {
      const int N = B.nym, nzm = B.nzm, nh = B.nymh, Pp = fft_y_pairs(B);
      const int groups = (nzm + 2 * Pp - 1) / (2 * Pp);
      const int k = lt / groups, i0 = (lt - k * groups) * 2 * Pp;
      double2 *cur = slot[it & 1];
      fft_tile<true, +1>(cur, N, ilog2(Pp), B.fft_y_radix, B.fft_y_np, tws, YInvSmemSrc{cur, N, nh, (N % 2) == 0},
                         YInvDst{B.phi + (long long)k * B.plane, N, nzm, i0});
    }
    fence_proxy_async_smem();
    __syncthreads();
  }
}

}  // namespace afid
