// Pressure Poisson solve of SolvePressureCorrection.F90:35-151 on one GPU:
//   y: real-to-complex FFT (two real rows packed in one complex line), fused
//      with the divergence of CalcLocalDivergence.F90 on its load;
//   z: complex FFT along kz on tiles of consecutive ky (in place);
//   x: one complex tridiagonal per (ky, kz), Thomas in dgttrf/dgttrs order;
//   then the inverse z and y transforms, the latter writing dph.
// The 2DECOMP pencil transposes of the reference disappear: each transform
// reads its lines directly from the plane-major layout.
//
// The FFTs are Stockham auto-sort passes of radix 4, 2, 3, 5 and 7 in shared
// memory, ping-ponging between two buffers.  Twiddles exp(-2 pi i n / N) come
// from a table computed on the host in extended precision and copied to
// shared memory by every block.
#pragma once
#include "afid_device.cuh"

namespace afid {

// radix-R butterfly on v[0..R-1] (unnormalised DFT, exponent sign ``sgn``)
template <int R>
__device__ __forceinline__ void dft_small(double2 (&v)[R], int sgn, const double2 *tw, int N) {
  if (R == 2) {
    const double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    const double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const double2 t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
    // w * t3 with w = sgn * i
    const double2 wt3 = make_double2(-sgn * t3.y, sgn * t3.x);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, wt3);
    v[3] = csub(t1, wt3);
  } else if (R == 3) {
    const double S3 = 0.86602540378443864676;   // sin(2 pi / 3)
    const double2 s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    const double2 a0 = v[0];
    const double2 m = make_double2(a0.x - 0.5 * s.x, a0.y - 0.5 * s.y);
    const double2 id = make_double2(-sgn * S3 * d.y, sgn * S3 * d.x);
    v[0] = cadd(a0, s);
    v[1] = cadd(m, id);
    v[2] = csub(m, id);
  } else if (R == 5) {
    const double C1 = 0.30901699437494742410, C2 = -0.80901699437494742410;
    const double S1 = 0.95105651629515357212, S2 = 0.58778525229247312917;
    const double2 a0 = v[0];
    const double2 s14 = cadd(v[1], v[4]), d14 = csub(v[1], v[4]);
    const double2 s23 = cadd(v[2], v[3]), d23 = csub(v[2], v[3]);
    const double2 r1 = make_double2(a0.x + C1 * s14.x + C2 * s23.x, a0.y + C1 * s14.y + C2 * s23.y);
    const double2 r2 = make_double2(a0.x + C2 * s14.x + C1 * s23.x, a0.y + C2 * s14.y + C1 * s23.y);
    const double2 q1 = make_double2(S1 * d14.x + S2 * d23.x, S1 * d14.y + S2 * d23.y);
    const double2 q2 = make_double2(S2 * d14.x - S1 * d23.x, S2 * d14.y - S1 * d23.y);
    // multiply by sgn * i
    const double2 iq1 = make_double2(-sgn * q1.y, sgn * q1.x);
    const double2 iq2 = make_double2(-sgn * q2.y, sgn * q2.x);
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

// One Stockham pass of radix R over L lines of length N, from buffer a into
// buffer b (both in shared memory).  LINE_MAJOR: element (l, n) at l*N + n,
// else at n*L + l.
constexpr int FFT_T = 256;          // threads per FFT block
constexpr int FFT_ELEMS = 3072;     // lines x N per block (two buffers: 96 KB)

template <int R, bool LINE_MAJOR>
__device__ __forceinline__ void stockham_pass(const double2 *__restrict__ a, double2 *__restrict__ b,
                                              int N, int L, int Ns, int sgn, const double2 *tw) {
  const int NR = N / R;
  const int tstr = N / (Ns * R);
  const int total = NR * L;
  for (int t = threadIdx.x; t < total; t += FFT_T) {
    int l, j;
    if (LINE_MAJOR) { j = t % NR; l = t / NR; } else { l = t % L; j = t / L; }
    const int k = j % Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = j + r * NR;
      v[r] = LINE_MAJOR ? a[l * N + n] : a[n * L + l];
    }
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        double2 w = tw[r * k * tstr];
        if (sgn > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dft_small<R>(v, sgn, tw, N);
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = base + r * Ns;
      if (LINE_MAJOR) b[l * N + n] = v[r]; else b[n * L + l] = v[r];
    }
  }
}

// Full transform; returns the buffer holding the result.
template <bool LINE_MAJOR>
__device__ double2 *stockham(double2 *a, double2 *b, int N, int L, const int *rad, int np,
                             int sgn, const double2 *tw) {
  int Ns = 1;
  for (int p = 0; p < np; ++p) {
    const int R = rad[p];
    switch (R) {
      case 4: stockham_pass<4, LINE_MAJOR>(a, b, N, L, Ns, sgn, tw); break;
      case 2: stockham_pass<2, LINE_MAJOR>(a, b, N, L, Ns, sgn, tw); break;
      case 3: stockham_pass<3, LINE_MAJOR>(a, b, N, L, Ns, sgn, tw); break;
      case 5: stockham_pass<5, LINE_MAJOR>(a, b, N, L, Ns, sgn, tw); break;
      default: stockham_pass<7, LINE_MAJOR>(a, b, N, L, Ns, sgn, tw); break;
    }
    __syncthreads();
    double2 *t = a; a = b; b = t;
    Ns *= R;
  }
  return a;
}

// Lines per block: row pairs of the y transforms, ky columns of the z
// transform.  Shared memory per block: two (lines x N) complex buffers plus
// the N twiddles.
__host__ __device__ __forceinline__ int fft_y_pairs(int nym) {
  int p = FFT_ELEMS / nym;
  if (p > 8) p = 8;
  if (p < 1) p = 1;
  return p;
}
__host__ __device__ __forceinline__ int fft_z_lines(int nzm) {
  int l = FFT_ELEMS / nzm;
  if (l > 16) l = 16;
  if (l < 1) l = 1;
  return l;
}
__host__ __device__ __forceinline__ int fft_smem_bytes(int n, int lines) {
  return (2 * lines + 1) * n * 16;
}

// ---------------------------------------------------------------------------
// y forward: rows (k, i) of length nym -> spec[k][i][ky], ky <= nym/2.
// FROM_VEL: the row values are the divergence of (vx, vy, vz) times 1/(al dt)
// computed on the fly; otherwise they are read from phi (the dph buffer).
// ---------------------------------------------------------------------------
template <bool FROM_VEL>
__global__ void __launch_bounds__(FFT_T, 2) k_fft_y_fwd(BatchDev bt, int ns) {
  extern __shared__ double2 fsm[];
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  const BoxScalars *S = B.sc;
  if (S->status != 0) return;
  const int N = B.nym, nzm = B.nzm;
  const int Pp = fft_y_pairs(N);
  const int groups = (nzm + 2 * Pp - 1) / (2 * Pp);
  const int tile = blockIdx.x - __ldg(bt.tile_off + b);
  const int k = tile / groups;
  const int i0 = (tile - k * groups) * 2 * Pp;
  double2 *a = fsm, *bb = fsm + Pp * N, *tws = fsm + 2 * Pp * N;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tws[t] = __ldg(B.twy + t);
  const long long P = B.plane;
  const double usdtal = FROM_VEL ? 1.0 / (S->dt * S->al) : 0.0;
  const double udx3m = FROM_VEL ? tabk(B, T_UDX3M, k) : 0.0;
  for (int t = threadIdx.x; t < 2 * Pp * N; t += blockDim.x) {
    const int row = t / N, j = t - row * N;
    const int i = i0 + row;
    double v = 0.0;
    if (i < nzm) {
      const long long o = (long long)k * P + (long long)i * N + j;
      if (FROM_VEL) {
        const int ip = i == nzm - 1 ? 0 : i + 1;
        const int jp = j == N - 1 ? 0 : j + 1;
        const double dq = (B.vz[(long long)k * P + (long long)ip * N + j] - B.vz[o]) * B.dz
                        + (B.vy[(long long)k * P + (long long)i * N + jp] - B.vy[o]) * B.dy
                        + (B.vx[o + P] - B.vx[o]) * udx3m;
        v = dq * usdtal;
      } else {
        v = B.phi[o];
      }
    }
    const int p = row >> 1;
    if (row & 1) a[p * N + j].y = v; else a[p * N + j].x = v;
  }
  __syncthreads();
  const double2 *r = stockham<true>(a, bb, N, Pp, B.fft_y_radix, B.fft_y_np, -1, tws);
  const int nh = B.nymh;
  for (int t = threadIdx.x; t < Pp * nh; t += blockDim.x) {
    const int p = t / nh, q = t - p * nh;
    const int i = i0 + 2 * p;
    if (i >= nzm) continue;
    const double2 z = r[p * N + q];
    const double2 zn = r[p * N + (q == 0 ? 0 : N - q)];
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
__global__ void __launch_bounds__(FFT_T, 2) k_fft_z(BatchDev bt, int ns, int sgn) {
  extern __shared__ double2 fsm[];
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  if (B.sc->status != 0) return;
  const int N = B.nzm, nh = B.nymh;
  const int L = fft_z_lines(N);
  const int ntl = (nh + L - 1) / L;
  const int tile = blockIdx.x - __ldg(bt.tile_off + b);
  const int k = tile / ntl;
  const int ky0 = (tile - k * ntl) * L;
  double2 *a = fsm, *bb = fsm + L * N, *tws = fsm + 2 * L * N;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tws[t] = __ldg(B.twz + t);
  double2 *spec = B.spec + (long long)k * N * nh;
  for (int t = threadIdx.x; t < L * N; t += blockDim.x) {
    const int l = t % L, n = t / L;
    const int ky = ky0 + l;
    a[n * L + l] = ky < nh ? spec[(long long)n * nh + ky] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const double2 *r = stockham<false>(a, bb, N, L, B.fft_z_radix, B.fft_z_np, sgn, tws);
  const double norm = (double)(B.nzm * B.nym);
  for (int t = threadIdx.x; t < L * N; t += blockDim.x) {
    const int l = t % L, n = t / L;
    const int ky = ky0 + l;
    if (ky < nh) {
      double2 v = r[n * L + l];
      if (sgn < 0) { v.x = v.x / norm; v.y = v.y / norm; }
      spec[(long long)n * nh + ky] = v;
    }
  }
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
  double2 *x = B.spec + m;
  double *dst = B.dstore + m;
  const long long st = nmode;
  const bool zero_mode = (ky == 0 && kz == 0);
  // forward elimination
  double s = 1.0 / ((__ldg(acph) - ak) - ak1);
  double d = 1.0;
  double2 y = x[0];
  y.x = y.x * s; y.y = y.y * s;
  double ap_prev = __ldg(apph) * s;
  x[0] = y;
  dst[0] = d;
  for (int k = 1; k < nxm; ++k) {
    s = 1.0 / ((__ldg(acph + k) - ak) - ak1);
    const double am = __ldg(amph + k) * s;
    const double fact = am / d;
    d = 1.0 - fact * ap_prev;
    double2 r = x[(long long)k * st];
    r.x = r.x * s; r.y = r.y * s;
    y.x = r.x - fact * y.x;
    y.y = r.y - fact * y.y;
    x[(long long)k * st] = y;
    dst[(long long)k * st] = d;
    ap_prev = __ldg(apph + k) * s;
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
  for (int k = nxm - 2; k >= 0; --k) {
    const double sk = 1.0 / ((__ldg(acph + k) - ak) - ak1);
    const double ap = __ldg(apph + k) * sk;
    const double dk = dst[(long long)k * st];
    const double2 yk = x[(long long)k * st];
    xn.x = (yk.x - ap * xn.x) / dk;
    xn.y = (yk.y - ap * xn.y) / dk;
    x[(long long)k * st] = xn;
  }
}

// ---------------------------------------------------------------------------
// y inverse (complex-to-real, unnormalised): spec[k][i][ky] -> phi[k][i][j].
// As in a c2r transform, the imaginary parts of the ky = 0 and ky = nym/2
// coefficients are ignored.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(FFT_T, 2) k_fft_y_inv(BatchDev bt, int ns) {
  extern __shared__ double2 fsm[];
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  if (B.sc->status != 0) return;
  const int N = B.nym, nzm = B.nzm, nh = B.nymh;
  const int Pp = fft_y_pairs(N);
  const int groups = (nzm + 2 * Pp - 1) / (2 * Pp);
  const int tile = blockIdx.x - __ldg(bt.tile_off + b);
  const int k = tile / groups;
  const int i0 = (tile - k * groups) * 2 * Pp;
  double2 *a = fsm, *bb = fsm + Pp * N, *tws = fsm + 2 * Pp * N;
  for (int t = threadIdx.x; t < N; t += blockDim.x) tws[t] = __ldg(B.twy + t);
  const bool even = (N % 2) == 0;
  for (int t = threadIdx.x; t < Pp * N; t += blockDim.x) {
    const int p = t / N, n = t - p * N;
    const int i = i0 + 2 * p;
    double2 A = make_double2(0.0, 0.0), Bv = make_double2(0.0, 0.0);
    const int q = n < nh ? n : N - n;
    const bool conj = n >= nh;
    const bool realonly = (q == 0) || (even && q == N / 2);
    if (i < nzm) {
      A = B.spec[((long long)k * nzm + i) * nh + q];
      if (realonly) A.y = 0.0; else if (conj) A.y = -A.y;
    }
    if (i + 1 < nzm) {
      Bv = B.spec[((long long)k * nzm + i + 1) * nh + q];
      if (realonly) Bv.y = 0.0; else if (conj) Bv.y = -Bv.y;
    }
    a[p * N + n] = make_double2(A.x - Bv.y, A.y + Bv.x);
  }
  __syncthreads();
  const double2 *r = stockham<true>(a, bb, N, Pp, B.fft_y_radix, B.fft_y_np, +1, tws);
  const long long P = B.plane;
  for (int t = threadIdx.x; t < 2 * Pp * N; t += blockDim.x) {
    const int row = t / N, j = t - row * N;
    const int i = i0 + row;
    if (i >= nzm) continue;
    const double2 z = r[(row >> 1) * N + j];
    B.phi[(long long)k * P + (long long)i * N + j] = (row & 1) ? z.y : z.x;
  }
}

}  // namespace afid
