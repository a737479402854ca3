// Pressure Poisson solve of SolvePressureCorrection.F90:35-151 on one GPU:
//   y: real-to-complex FFT (two real rows packed in one complex line) of dph;
//   z: complex FFT along kz on tiles of consecutive ky (in place);
//   x: one complex tridiagonal per (ky, kz), Thomas in dgttrf/dgttrs order;
//   then the inverse z and y transforms, the latter writing dph.
// The 2DECOMP pencil transposes of the reference disappear: each transform
// reads its lines directly from the plane-major layout.
//
// The FFTs are Stockham auto-sort passes of radix 16, 8, 4, 2, 3, 5 and 7
// (plans in increasing radix order, e.g. 768 = 3 x 16 x 16): the first pass
// streams from global memory, the inner passes run in place in shared memory
// and the last pass of the z and inverse-y transforms streams back to global
// memory.  Twiddles exp(-2 pi i n / N) come from a table computed on the host
// in extended precision and copied to shared memory by every block.
#pragma once
#include "afid_device.cuh"

namespace afid {

// radix-R butterfly on v[0..R-1] (unnormalised DFT, exponent sign ``sgn``)
__device__ __forceinline__ double2 cmul_wi(double2 a, double c, double s, int sgn) {
  // a * (c + i sgn s)
  const double ss = sgn > 0 ? s : -s;
  return make_double2(a.x * c - a.y * ss, a.x * ss + a.y * c);
}
__device__ __forceinline__ double2 mul_sgn_i(double2 a, int sgn) {   // a * (sgn i)
  return make_double2(-sgn * a.y, sgn * a.x);
}
__device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2, double2 &a3, int sgn) {
  const double2 t0 = cadd(a0, a2), t1 = csub(a0, a2);
  const double2 t2 = cadd(a1, a3), t3 = csub(a1, a3);
  const double2 wt3 = mul_sgn_i(t3, sgn);
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, wt3);
  a3 = csub(t1, wt3);
}

template <int R>
__device__ __forceinline__ void dft_small(double2 (&v)[R], int sgn, const double2 *tw, int N) {
  constexpr double H = 0.70710678118654752440;    // cos(pi/4)
  constexpr double C8 = 0.92387953251128675613;   // cos(pi/8)
  constexpr double S8 = 0.38268343236508977173;   // sin(pi/8)
  if constexpr (R == 2) {
    const double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    dft4(v[0], v[1], v[2], v[3], sgn);
  } else if constexpr (R == 8) {
    // 8 = 2 x 4: four-point DFTs over n2 of x[n1 + 2 n2], twiddle W8^(n1 k2),
    // two-point DFTs over n1; X[4 k1 + k2]
    double2 a0 = v[0], a1 = v[2], a2 = v[4], a3 = v[6];
    double2 b0 = v[1], b1 = v[3], b2 = v[5], b3 = v[7];
    dft4(a0, a1, a2, a3, sgn);
    dft4(b0, b1, b2, b3, sgn);
    b1 = cmul_wi(b1, H, H, sgn);
    b2 = mul_sgn_i(b2, sgn);
    b3 = cmul_wi(b3, -H, H, sgn);
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
    for (int n1 = 0; n1 < 4; ++n1) dft4(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12], sgn);
    v[5] = cmul_wi(v[5], C8, S8, sgn);        // n1=1 k2=1: m=1
    v[9] = cmul_wi(v[9], H, H, sgn);          // n1=1 k2=2: m=2
    v[13] = cmul_wi(v[13], S8, C8, sgn);      // n1=1 k2=3: m=3
    v[6] = cmul_wi(v[6], H, H, sgn);          // n1=2 k2=1: m=2
    v[10] = mul_sgn_i(v[10], sgn);            // n1=2 k2=2: m=4
    v[14] = cmul_wi(v[14], -H, H, sgn);       // n1=2 k2=3: m=6
    v[7] = cmul_wi(v[7], S8, C8, sgn);        // n1=3 k2=1: m=3
    v[11] = cmul_wi(v[11], -H, H, sgn);       // n1=3 k2=2: m=6
    v[15] = cmul_wi(v[15], -C8, -S8, sgn);    // n1=3 k2=3: m=9
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) dft4(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3], sgn);
    // X[4 k1 + k2] = v[4 k2 + k1]: transpose the 4 x 4 index grid
    double2 t;
    t = v[1]; v[1] = v[4]; v[4] = t;
    t = v[2]; v[2] = v[8]; v[8] = t;
    t = v[3]; v[3] = v[12]; v[12] = t;
    t = v[6]; v[6] = v[9]; v[9] = t;
    t = v[7]; v[7] = v[13]; v[13] = t;
    t = v[11]; v[11] = v[14]; v[14] = t;
  } else if constexpr (R == 3) {
    const double S3 = 0.86602540378443864676;   // sin(2 pi / 3)
    const double2 s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    const double2 a0 = v[0];
    const double2 m = make_double2(a0.x - 0.5 * s.x, a0.y - 0.5 * s.y);
    const double2 id = make_double2(-sgn * S3 * d.y, sgn * S3 * d.x);
    v[0] = cadd(a0, s);
    v[1] = cadd(m, id);
    v[2] = csub(m, id);
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
    const double2 iq1 = mul_sgn_i(q1, sgn);
    const double2 iq2 = mul_sgn_i(q2, sgn);
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
        if (sgn > 0) w.y = -w.y;
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
// Every pass streams from a source functor to a destination functor: the
// first pass reads global memory, inner passes go between two shared
// buffers, and the last pass of the z and inverse-y transforms writes global
// memory.  LINE_MAJOR: element (l, n) at l*N + n, else at n*L + l.
constexpr int FFT_T = 256;    // threads per FFT block

template <bool LM>
__device__ __forceinline__ void bfly_index(int t, int NR, int L, int &l, int &j) {
  if (LM) { j = t % NR; l = t / NR; } else { l = t % L; j = t / L; }
}
template <bool LM>
__device__ __forceinline__ int sidx(int l, int n, int N, int L) { return LM ? l * N + n : n * L + l; }

template <int R>
__device__ __forceinline__ void twiddle(double2 (&v)[R], int k, int tstr, int sgn, const double2 *tw) {
#pragma unroll
  for (int r = 1; r < R; ++r) {
    double2 w = tw[r * k * tstr];
    if (sgn > 0) w.y = -w.y;
    v[r] = cmul(v[r], w);
  }
}

template <int R, bool LM, class Src, class Dst>
__device__ __forceinline__ void pass_stream(int N, int L, int Ns, int sgn, const double2 *tw,
                                            const Src &src, const Dst &dst) {
  const int NR = N / R, tstr = N / (Ns * R), total = NR * L;
  for (int t = threadIdx.x; t < total; t += FFT_T) {
    int l, j;
    bfly_index<LM>(t, NR, L, l, j);
    const int k = j % Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src(l, j + r * NR);
    if (Ns > 1) twiddle<R>(v, k, tstr, sgn, tw);
    dft_small<R>(v, sgn, tw, N);
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst(l, base + r * Ns, v[r]);
  }
}

template <bool LM, class Src, class Dst>
__device__ __forceinline__ void run_stream(int R, int N, int L, int Ns, int sgn, const double2 *tw,
                                           const Src &src, const Dst &dst) {
  switch (R) {
    case 16: pass_stream<16, LM>(N, L, Ns, sgn, tw, src, dst); break;
    case 8: pass_stream<8, LM>(N, L, Ns, sgn, tw, src, dst); break;
    case 4: pass_stream<4, LM>(N, L, Ns, sgn, tw, src, dst); break;
    case 2: pass_stream<2, LM>(N, L, Ns, sgn, tw, src, dst); break;
    case 3: pass_stream<3, LM>(N, L, Ns, sgn, tw, src, dst); break;
    case 5: pass_stream<5, LM>(N, L, Ns, sgn, tw, src, dst); break;
    default: pass_stream<7, LM>(N, L, Ns, sgn, tw, src, dst); break;
  }
}

template <bool LM>
struct SmemDst {
  double2 *a; int N, L;
  __device__ __forceinline__ void operator()(int l, int n, double2 v) const { a[sidx<LM>(l, n, N, L)] = v; }
};
template <bool LM>
struct SmemSrc {
  const double2 *a; int N, L;
  __device__ __forceinline__ double2 operator()(int l, int n) const { return a[sidx<LM>(l, n, N, L)]; }
};

// Transform of L lines.  The first pass streams from ``src`` into shared
// buffer a; inner passes ping-pong between a and b; the last pass streams to
// ``dst`` when LAST_TO_DST, otherwise it lands in shared memory too.  Returns
// the shared buffer holding the result (meaningful when !LAST_TO_DST).
template <bool LM, bool LAST_TO_DST, class Src, class Dst>
__device__ double2 *fft_lines(double2 *a, double2 *b, int N, int L, const int *rad, int np, int sgn,
                              const double2 *tw, const Src &src, const Dst &dst) {
  if (np == 1 && LAST_TO_DST) {
    run_stream<LM>(rad[0], N, L, 1, sgn, tw, src, dst);
    return a;
  }
  run_stream<LM>(rad[0], N, L, 1, sgn, tw, src, SmemDst<LM>{a, N, L});
  __syncthreads();
  int Ns = rad[0];
  const int nin = LAST_TO_DST ? np - 1 : np;
  for (int p = 1; p < nin; ++p) {
    run_stream<LM>(rad[p], N, L, Ns, sgn, tw, SmemSrc<LM>{a, N, L}, SmemDst<LM>{b, N, L});
    __syncthreads();
    double2 *t = a; a = b; b = t;
    Ns *= rad[p];
  }
  if (LAST_TO_DST) run_stream<LM>(rad[np - 1], N, L, Ns, sgn, tw, SmemSrc<LM>{a, N, L}, dst);
  return a;
}

// Transform of L lines whose input is already in shared buffer a: every
// pass goes shared -> shared (a, b alternating) except the last, which goes
// to ``dst`` when LAST_TO_DST.  Returns the buffer holding the result
// (meaningful when !LAST_TO_DST).
template <bool LM, bool LAST_TO_DST, class Dst>
__device__ double2 *fft_lines_smem(double2 *a, double2 *b, int N, int L, const int *rad, int np, int sgn,
                                   const double2 *tw, const Dst &dst, int Ns0 = 1) {
  int Ns = Ns0;
  const int nin = LAST_TO_DST ? np - 1 : np;
  for (int p = 0; p < nin; ++p) {
    run_stream<LM>(rad[p], N, L, Ns, sgn, tw, SmemSrc<LM>{a, N, L}, SmemDst<LM>{b, N, L});
    __syncthreads();
    double2 *t = a; a = b; b = t;
    Ns *= rad[p];
  }
  if (LAST_TO_DST) run_stream<LM>(rad[np - 1], N, L, Ns, sgn, tw, SmemSrc<LM>{a, N, L}, dst);
  return a;
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(src));
}
__device__ __forceinline__ void cp_async8d(void *dst, const void *src) {
  unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(saddr), "l"(src));
}
__device__ __forceinline__ void cp_async_commit_wait() {
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_all;\n" ::);
}

// Lines per block and shared memory: two (lines x N) buffers when the
// transform has a pass between two shared-memory stages, otherwise one, plus
// the N twiddles; lines are capped so that a block stays within ~100 KB.
__host__ __device__ __forceinline__ int fft_nbuf(int np, bool last_to_dst) {
  // the copied-in tile plus one buffer per pass that writes shared memory,
  // ping-ponging: two buffers unless the only pass streams straight out
  const int smem_stages = last_to_dst ? np - 1 : np;
  return smem_stages >= 1 ? 2 : 1;
}
__host__ __device__ __forceinline__ int fft_lines_per_block(int N, int nbuf, int cap) {
  int l = (100 * 1024) / (16 * N * nbuf);
  if (l > cap) l = cap;
  return l < 1 ? 1 : l;
}
__host__ __device__ __forceinline__ int fft_y_pairs(const BoxDev &B) {
  if (B.fy_lines > 0) return B.fy_lines;
  return fft_lines_per_block(B.nym, fft_nbuf(B.fft_y_np, false), 16);
}
__host__ __device__ __forceinline__ int fft_z_lines(const BoxDev &B) {
  const int l = B.fz_lines > 0 ? B.fz_lines : fft_lines_per_block(B.nzm, fft_nbuf(B.fft_z_np, true), 16);
  return l < B.nymh ? l : B.nymh;
}
// largest admissible tuning values (shared memory of one block <= 200 KB)
__host__ __device__ __forceinline__ int fft_max_lines(int N, int nbuf) {
  return (200 * 1024) / (16 * N * nbuf) - 1;
}
__host__ __device__ __forceinline__ int fft_y_smem(const BoxDev &B) {
  // forward: lines + copied-in rows + twiddles; inverse: lines + raw
  // half-spectrum rows (2 Pp (nym/2+1) complex) + twiddles
  const int Pp = fft_y_pairs(B);
  return ((2 * Pp + 1) * B.nym + 2 * Pp) * 16;
}
__host__ __device__ __forceinline__ int fft_z_smem(const BoxDev &B) {
  return (fft_nbuf(B.fft_z_np, true) * fft_z_lines(B) + 1) * B.nzm * 16;
}

// ---------------------------------------------------------------------------
// y forward: rows (k, i) of length nym of dph -> spec[k][i][ky], ky <= nym/2.
// ---------------------------------------------------------------------------
struct NoDst {
  __device__ __forceinline__ void operator()(int, int, double2) const {}
};

// y forward over the rows of dph (phi): the 2*Pp rows of the block are
// copied into shared memory with cp.async, packed two by two as complex
// lines, transformed, and unpacked into the half spectrum.
__global__ void __launch_bounds__(FFT_T, 2) k_fft_y_fwd(BatchDev bt, int ns) {
  extern __shared__ double2 fsm[];
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  const BoxScalars *S = B.sc;
  if (S->status != 0) return;
  const int N = B.nym, nzm = B.nzm;
  const int Pp = fft_y_pairs(B);
  const int groups = (nzm + 2 * Pp - 1) / (2 * Pp);
  const int tile = blockIdx.x - __ldg(bt.tile_off + b);
  const int k = tile / groups;
  const int i0 = (tile - k * groups) * 2 * Pp;
  double2 *a = fsm, *bb = fsm + Pp * N, *tws = fsm + 2 * Pp * N;
  // copy in: row r of the block (i = i0 + r) as doubles into bb; line p is
  // the complex pair (row 2p, row 2p+1), re-read below as double2 from a
  double *rows = (double *)bb;
  const double *phik = B.phi + (long long)k * B.plane;
  for (int t = threadIdx.x; t < 2 * Pp * N; t += FFT_T) {
    const int r = t / N, j = t - r * N;
    if (i0 + r < nzm) cp_async8d(rows + r * N + j, phik + (long long)(i0 + r) * N + j);
    else rows[r * N + j] = 0.0;
  }
  for (int t = threadIdx.x; t < N; t += FFT_T) tws[t] = __ldg(B.twy + t);
  cp_async_commit_wait();
  __syncthreads();
  for (int t = threadIdx.x; t < Pp * N; t += FFT_T) {
    const int p = t / N, j = t - p * N;
    a[p * N + j] = make_double2(rows[2 * p * N + j], rows[(2 * p + 1) * N + j]);
  }
  __syncthreads();
  a = fft_lines_smem<true, false>(a, bb, N, Pp, B.fft_y_radix, B.fft_y_np, -1, tws, NoDst{});
  // unpack the two real transforms: A = (Z_q + conj Z_{N-q}) / 2,
  // B = (Z_q - conj Z_{N-q}) / (2i)
  const int nh = B.nymh;
  for (int t = threadIdx.x; t < Pp * nh; t += FFT_T) {
    const int p = t / nh, q = t - p * nh;
    const int i = i0 + 2 * p;
    if (i >= nzm) continue;
    const double2 z = a[p * N + q];
    const double2 zn = a[p * N + (q == 0 ? 0 : N - q)];
    const double2 A = make_double2((z.x + zn.x) * 0.5, (z.y - zn.y) * 0.5);
    const double2 Bv = make_double2((z.y + zn.y) * 0.5, (zn.x - z.x) * 0.5);
    const long long base = ((long long)k * nzm + i) * nh + q;
    B.spec[base] = A;
    if (i + 1 < nzm) B.spec[base + nh] = Bv;
  }
}

// ---------------------------------------------------------------------------
// z transform in place on spec[k][kz][ky] for a tile of L consecutive ky.
// Forward transforms divide by nym*nzm (SolvePressureCorrection.F90:105).
// ---------------------------------------------------------------------------
struct ZSrc {
  const double2 *spec; int nh, ky0;
  __device__ __forceinline__ double2 operator()(int l, int n) const {
    const int ky = ky0 + l;
    return ky < nh ? spec[(long long)n * nh + ky] : make_double2(0.0, 0.0);
  }
};
struct ZDst {
  double2 *spec; int nh, ky0; double norm; bool scale;
  __device__ __forceinline__ void operator()(int l, int n, double2 v) const {
    const int ky = ky0 + l;
    if (ky >= nh) return;
    if (scale) { v.x = v.x / norm; v.y = v.y / norm; }
    spec[(long long)n * nh + ky] = v;
  }
};

__global__ void __launch_bounds__(FFT_T, 2) k_fft_z(BatchDev bt, int ns, int sgn) {
  extern __shared__ double2 fsm[];
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  if (B.sc->status != 0) return;
  const int N = B.nzm, nh = B.nymh;
  const int L = fft_z_lines(B);
  const int ntl = (nh + L - 1) / L;
  const int tile = blockIdx.x - __ldg(bt.tile_off + b);
  const int k = tile / ntl;
  const int ky0 = (tile - k * ntl) * L;
  const int nb = fft_nbuf(B.fft_z_np, true);
  double2 *a = fsm, *bb = fsm + (nb - 1) * L * N, *tws = fsm + nb * L * N;
  double2 *spec = B.spec + (long long)k * N * nh;
  for (int t = threadIdx.x; t < L * N; t += FFT_T) {
    const int l = t % L, n = t / L;
    if (ky0 + l < nh) cp_async16(a + n * L + l, spec + (long long)n * nh + ky0 + l);
    else a[n * L + l] = make_double2(0.0, 0.0);
  }
  for (int t = threadIdx.x; t < N; t += FFT_T) tws[t] = __ldg(B.twz + t);
  cp_async_commit_wait();
  __syncthreads();
  fft_lines_smem<false, true>(a, bb, N, L, B.fft_z_radix, B.fft_z_np, sgn, tws,
                              ZDst{spec, nh, ky0, (double)(B.nzm * B.nym), sgn < 0});
}

// ---------------------------------------------------------------------------
// x: complex tridiagonal per mode (SolvePressureCorrection.F90:117-137), one
// thread per (ky, kz), marching k.  Row k of the normalised system is
//   amph(k) x(k-1) + x(k) + apph(k) x(k+1) = dphc(k) s(k),
//   s(k) = 1 / (acphk(k) - ak2(ky) - ak1(kz)).
// Its coefficients are real, so the complex Thomas sweep is a real sweep
// applied to both parts.  The (0,0) mode is singular (Neumann in x): its
// last equation is dropped and its last unknown set to zero.
// ---------------------------------------------------------------------------
constexpr int KP_U = 4;   // planes per prefetch chunk of the sweeps

__global__ void __launch_bounds__(256) k_poisson_x(BatchDev bt, int ns) {
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  if (B.sc->status != 0) return;
  const int nh = B.nymh, nzm = B.nzm, nxm = B.nxm;
  const long long m = (long long)(blockIdx.x - __ldg(bt.tile_off + b)) * blockDim.x + threadIdx.x;
  const long long nmode = (long long)nzm * nh;
  if (m >= nmode) return;
  const int kz = (int)(m / nh), ky = (int)(m - (long long)kz * nh);
  const double ak = __ldg(B.tab + (long long)T_NK * B.nx + nzm + ky);   // ak2(ky)
  const double ak1 = __ldg(B.tab + (long long)T_NK * B.nx + kz);      // ak1(kz)
  const double *amph = B.tab + (long long)T_AMPHK * B.nx;
  const double *acph = B.tab + (long long)T_ACPHK * B.nx;
  const double *apph = B.tab + (long long)T_APPHK * B.nx;
  double2 *__restrict__ x = B.spec + m;
  double *__restrict__ dst = B.dstore + m;
  const long long st = nmode;
  const bool zero_mode = (ky == 0 && kz == 0);
  // forward elimination (dgttrf + dgttrs forward sweep), planes in chunks
  double d = 1.0, ap_prev = 0.0;
  double2 y = make_double2(0.0, 0.0);
  for (int k0 = 0; k0 < nxm; k0 += KP_U) {
    double2 r[KP_U];
#pragma unroll
    for (int u = 0; u < KP_U; ++u)
      if (k0 + u < nxm) r[u] = x[(long long)(k0 + u) * st];
#pragma unroll
    for (int u = 0; u < KP_U; ++u) {
      const int k = k0 + u;
      if (k >= nxm) break;
      const double s = 1.0 / ((__ldg(acph + k) - ak) - ak1);
      double2 rk = r[u];
      rk.x = rk.x * s; rk.y = rk.y * s;
      if (k == 0) {
        y = rk;
      } else {
        const double am = __ldg(amph + k) * s;
        const double fact = am / d;
        d = 1.0 - fact * ap_prev;
        y.x = rk.x - fact * y.x;
        y.y = rk.y - fact * y.y;
      }
      x[(long long)k * st] = y;
      dst[(long long)k * st] = d;
      ap_prev = __ldg(apph + k) * s;
    }
  }
  // back substitution
  double2 xn;
  if (zero_mode) {
    xn = make_double2(0.0, 0.0);
  } else {
    xn.x = y.x / d;
    xn.y = y.y / d;
  }
  x[(long long)(nxm - 1) * st] = xn;
  for (int k0 = nxm - 2; k0 >= 0; k0 -= KP_U) {
    double2 yk[KP_U];
    double dk[KP_U];
#pragma unroll
    for (int u = 0; u < KP_U; ++u) {
      const int k = k0 - u;
      if (k >= 0) { yk[u] = x[(long long)k * st]; dk[u] = dst[(long long)k * st]; }
    }
#pragma unroll
    for (int u = 0; u < KP_U; ++u) {
      const int k = k0 - u;
      if (k < 0) break;
      const double sk = 1.0 / ((__ldg(acph + k) - ak) - ak1);
      const double ap = __ldg(apph + k) * sk;
      xn.x = (yk[u].x - ap * xn.x) / dk[u];
      xn.y = (yk[u].y - ap * xn.y) / dk[u];
      x[(long long)k * st] = xn;
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
    if (i < nzm) phi[(long long)i * N + j] = v.x;
    if (i + 1 < nzm) phi[(long long)(i + 1) * N + j] = v.y;
  }
};

// y inverse (complex-to-real, unnormalised): spec[k][i][ky] -> phi[k][i][j].
// As in a c2r transform, the imaginary parts of the ky = 0 and ky = nym/2
// coefficients are ignored.  The block's half-spectrum rows are copied into
// shared memory with cp.async; two rows are recovered from one complex line
// Z = A + i B.  The raw rows' buffer becomes the second ping-pong buffer once
// the first pass has read it.
__global__ void __launch_bounds__(FFT_T, 2) k_fft_y_inv(BatchDev bt, int ns) {
  extern __shared__ double2 fsm[];
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  if (B.sc->status != 0) return;
  const int N = B.nym, nzm = B.nzm, nh = B.nymh;
  const int Pp = fft_y_pairs(B);
  const int groups = (nzm + 2 * Pp - 1) / (2 * Pp);
  const int tile = blockIdx.x - __ldg(bt.tile_off + b);
  const int k = tile / groups;
  const int i0 = (tile - k * groups) * 2 * Pp;
  // layout: a = Pp*N, raw (= b) = 2*Pp*nh >= Pp*N, twiddles
  double2 *a = fsm, *raw = fsm + Pp * N, *tws = raw + 2 * Pp * nh;
  const double2 *speck = B.spec + (long long)k * nzm * nh;
  for (int t = threadIdx.x; t < 2 * Pp * nh; t += FFT_T) {
    const int r = t / nh, q = t - r * nh;
    if (i0 + r < nzm) cp_async16(raw + t, speck + (long long)(i0 + r) * nh + q);
    else raw[t] = make_double2(0.0, 0.0);
  }
  for (int t = threadIdx.x; t < N; t += FFT_T) tws[t] = __ldg(B.twy + t);
  cp_async_commit_wait();
  __syncthreads();
  const int np = B.fft_y_np;
  YInvDst dst{B.phi + (long long)k * B.plane, N, nzm, i0};
  const YInvSmemSrc src{raw, N, nh, (N % 2) == 0};
  if (np == 1) {
    run_stream<true>(B.fft_y_radix[0], N, Pp, 1, +1, tws, src, dst);
    return;
  }
  run_stream<true>(B.fft_y_radix[0], N, Pp, 1, +1, tws, src, SmemDst<true>{a, N, Pp});
  __syncthreads();
  fft_lines_smem<true, true>(a, raw, N, Pp, B.fft_y_radix + 1, np - 1, +1, tws, dst, B.fft_y_radix[0]);
}

}  // namespace afid
