// Explicit advection/diffusion terms, Crank-Nicolson right-hand sides and the
// x-direction tridiagonal solves of one RK3 substep, plus the projection
// (CorrectVelocity + CorrectPressure) and the per-step reductions.
//
// Arithmetic follows the reference expression by expression; the library is
// compiled without FMA contraction so that every stencil value is the same
// IEEE result the reference's x86-64 build computes for the same inputs.
#pragma once
#include "afid_device.cuh"

namespace afid {

enum FieldId { F_VX = 0, F_VY = 1, F_VZ = 2, F_T = 3, F_PR = 4, F_NF = 5 };

struct StencilConst {
  double udy, udz;           // dy/4, dz/4
  double udyq_re, udzq_re;   // dyq/ren, dzq/ren
  double udyq_pe, udzq_pe;   // dyq/pec, dzq/pec
};

__device__ __forceinline__ StencilConst make_sconst(const BoxDev &B) {
  StencilConst c;
  c.udy = B.dy * 0.25;
  c.udz = B.dz * 0.25;
  c.udyq_re = B.dyq / B.ren;
  c.udzq_re = B.dzq / B.ren;
  c.udyq_pe = B.dyq / B.pec;
  c.udzq_pe = B.dzq / B.pec;
  return c;
}

// ---------------------------------------------------------------------------
// The four explicit terms.  ``a(f, dk, dj, di)`` returns field f at
// (k+dk, j+dj, i+di) around the point being computed; dk is -1, 0 or +1.
// ``dkm``/``dkp`` are kmv(kc)-kc and kpv(kc)-kc (0 at the walls).
// ---------------------------------------------------------------------------
// ExplicitTermsVX.F90:55-101 (k = 2..nxm)
template <class A>
__device__ __forceinline__ double h_vx(const A &a, const StencilConst &c, double udx3c_k) {
  const double vxc = a(F_VX, 0, 0, 0);
  double hxz = (((a(F_VZ, 0, 0, 1) + a(F_VZ, -1, 0, 1)) * (a(F_VX, 0, 0, 1) + vxc))
                - ((a(F_VZ, 0, 0, 0) + a(F_VZ, -1, 0, 0)) * (vxc + a(F_VX, 0, 0, -1)))) * c.udz;
  double hxy = (((a(F_VY, 0, 1, 0) + a(F_VY, -1, 1, 0)) * (a(F_VX, 0, 1, 0) + vxc))
                - ((a(F_VY, 0, 0, 0) + a(F_VY, -1, 0, 0)) * (vxc + a(F_VX, 0, -1, 0)))) * c.udy;
  const double p = a(F_VX, 1, 0, 0) + vxc;
  const double m = vxc + a(F_VX, -1, 0, 0);
  double hxx = (p * p - m * m) * udx3c_k * 0.25;
  double tempit = a(F_T, 0, 0, 0);
  double dzzvx = (a(F_VX, 0, 0, -1) - 2.0 * vxc + a(F_VX, 0, 0, 1)) * c.udzq_re;
  double dyyvx = (a(F_VX, 0, -1, 0) - 2.0 * vxc + a(F_VX, 0, 1, 0)) * c.udyq_re;
  return -(hxx + hxy + hxz) + dyyvx + dzzvx + tempit;
}

// ExplicitTermsVY.F90:54-98 (k = 1..nxm)
template <class A>
__device__ __forceinline__ double h_vy(const A &a, const StencilConst &c, double udx3m_k, int dkm, int dkp) {
  const double vyc = a(F_VY, 0, 0, 0);
  double hyx = ((a(F_VX, 1, 0, 0) + a(F_VX, 1, -1, 0)) * (a(F_VY, dkp, 0, 0) + vyc)
                - (a(F_VX, 0, 0, 0) + a(F_VX, 0, -1, 0)) * (vyc + a(F_VY, dkm, 0, 0))) * udx3m_k * 0.25;
  const double p = a(F_VY, 0, 1, 0) + vyc;
  const double m = a(F_VY, 0, -1, 0) + vyc;
  double hyy = (p * p - m * m) * c.udy;
  double hyz = ((a(F_VY, 0, 0, 1) + vyc) * (a(F_VZ, 0, 0, 1) + a(F_VZ, 0, -1, 1))
                - (vyc + a(F_VY, 0, 0, -1)) * (a(F_VZ, 0, 0, 0) + a(F_VZ, 0, -1, 0))) * c.udz;
  double dyyvy = (a(F_VY, 0, 1, 0) - 2.0 * vyc + a(F_VY, 0, -1, 0)) * c.udyq_re;
  double dzzvy = (a(F_VY, 0, 0, 1) - 2.0 * vyc + a(F_VY, 0, 0, -1)) * c.udzq_re;
  return -(hyx + hyy + hyz) + dyyvy + dzzvy;
}

// ExplicitTermsVZ.F90:56-101 (k = 1..nxm)
template <class A>
__device__ __forceinline__ double h_vz(const A &a, const StencilConst &c, double udx3m_k, int dkm, int dkp) {
  const double vzc = a(F_VZ, 0, 0, 0);
  const double p = a(F_VZ, 0, 0, 1) + vzc;
  const double m = a(F_VZ, 0, 0, -1) + vzc;
  double hzz = (p * p - m * m) * c.udz;
  double hzy = ((a(F_VY, 0, 1, 0) + a(F_VY, 0, 1, -1)) * (a(F_VZ, 0, 1, 0) + vzc)
                - (a(F_VY, 0, 0, 0) + a(F_VY, 0, 0, -1)) * (vzc + a(F_VZ, 0, -1, 0))) * c.udy;
  double hzx = ((a(F_VX, 1, 0, 0) + a(F_VX, 1, 0, -1)) * (a(F_VZ, dkp, 0, 0) + vzc)
                - (a(F_VX, 0, 0, 0) + a(F_VX, 0, 0, -1)) * (vzc + a(F_VZ, dkm, 0, 0))) * udx3m_k * 0.25;
  double dzzvz = (a(F_VZ, 0, 0, 1) - 2.0 * vzc + a(F_VZ, 0, 0, -1)) * c.udzq_re;
  double dyyvz = (a(F_VZ, 0, 1, 0) - 2.0 * vzc + a(F_VZ, 0, -1, 0)) * c.udyq_re;
  return -(hzx + hzy + hzz) + dyyvz + dzzvz;
}

// ExplicitTermsTemp.F90:52-93 (k = 2..nxm)
template <class A>
__device__ __forceinline__ double h_temp(const A &a, const StencilConst &c, double udx3c_k) {
  const double tc = a(F_T, 0, 0, 0);
  double htz = ((a(F_VZ, -1, 0, 1) + a(F_VZ, 0, 0, 1)) * (a(F_T, 0, 0, 1) + tc)
                - (a(F_VZ, -1, 0, 0) + a(F_VZ, 0, 0, 0)) * (tc + a(F_T, 0, 0, -1))) * c.udz;
  double hty = ((a(F_VY, 0, 1, 0) + a(F_VY, -1, 1, 0)) * (a(F_T, 0, 1, 0) + tc)
                - (a(F_VY, 0, 0, 0) + a(F_VY, -1, 0, 0)) * (tc + a(F_T, 0, -1, 0))) * c.udy;
  double htx = ((a(F_VX, 1, 0, 0) + a(F_VX, 0, 0, 0)) * (a(F_T, 1, 0, 0) + tc)
                - (a(F_VX, 0, 0, 0) + a(F_VX, -1, 0, 0)) * (tc + a(F_T, -1, 0, 0))) * udx3c_k * 0.25;
  double dzzt = (a(F_T, 0, 0, 1) - 2.0 * tc + a(F_T, 0, 0, -1)) * c.udzq_pe;
  double dyyt = (a(F_T, 0, 1, 0) - 2.0 * tc + a(F_T, 0, -1, 0)) * c.udyq_pe;
  return -(htx + hty + htz) + dyyt + dzzt;
}

// Implicit right-hand sides (ImplicitAndUpdate*.F90).  Returned value is the
// unscaled rhs; the caller multiplies by the row scale of the solver.
// ImplicitAndUpdateVX.F90:40-58
__device__ __forceinline__ double rhs_vx(double H, double Hold, double vxp, double vxc, double vxm,
                                         double prc, double prm, double am, double ac, double ap,
                                         double al, double ga, double ro, double alre, double dt,
                                         double udx3c_k) {
  const double udx3 = al * udx3c_k;
  const double dxx = vxp * ap + vxc * ac + vxm * am;
  const double dxp = (prc - prm) * udx3;
  return (ga * H + ro * Hold + alre * dxx - dxp) * dt;
}
// ImplicitAndUpdateVY.F90:52-63 / ImplicitAndUpdateVZ.F90:48-59; ``dp`` is
// the pressure-gradient term already formed by the caller.
__device__ __forceinline__ double rhs_vyz(double H, double Hold, double qp, double qc, double qm,
                                          double am, double ac, double ap, double dp,
                                          double ga, double ro, double alre, double dt) {
  const double dxx = qp * ap + qc * ac + qm * am;
  return (ga * H + ro * Hold + alre * dxx - dp) * dt;
}
// ImplicitAndUpdateTemp.F90:41-49
__device__ __forceinline__ double rhs_temp(double H, double Hold, double tp, double tc, double tm,
                                           double am, double ac, double ap,
                                           double ga, double ro, double alpec, double dt) {
  const double dxx = tp * ap + tc * ac + tm * am;
  return (ga * H + ro * Hold + alpec * dxx) * dt;
}

__device__ __forceinline__ const double *coefp(const BoxDev &B, int sys, int arr) {
  return B.coef + (long long)(sys * C_N + arr) * B.nx;
}

// ---------------------------------------------------------------------------
// Per-substep preparation: coefficients al/ga/ro/beta and the LU factors of
// the three x-tridiagonal matrices (SolveImpEqnUpdate_X.F90:25-44,
// SolveImpEqnUpdate_YZ.F90:25-38, SolveImpEqnUpdate_Temp.F90:25-47), in the
// dgttrf operation order without pivoting (the matrices are diagonally
// dominant; a pivot that LAPACK would take is reported as status -2).
// One block per box.
// ---------------------------------------------------------------------------
__global__ void k_substep_prep(const BoxDev *__restrict__ boxes, int nbox, int ns) {
  const int b = blockIdx.x;
  if (b >= nbox) return;
  const BoxDev &B = boxes[b];
  if (!B.active || ns >= B.nsst) return;
  BoxScalars *S = B.sc;
  if (S->status != 0) return;
  __shared__ double s_bx[3];
  if (threadIdx.x == 0) {
    double gam[3], rom[3];
    if (B.nsst > 1) {
      gam[0] = 8.0 / 15.0; gam[1] = 5.0 / 12.0; gam[2] = 3.0 / 4.0;
      rom[0] = 0.0; rom[1] = -17.0 / 60.0; rom[2] = -5.0 / 12.0;
    } else {
      gam[0] = 1.5; gam[1] = 0.0; gam[2] = 0.0;
      rom[0] = -0.5; rom[1] = 0.0; rom[2] = 0.0;
    }
    const double dt = S->dt;
    const double al = gam[ns] + rom[ns];
    const double beta = dt / B.ren * 0.5;     // TimeMarcher.F90:22
    S->al = al; S->ga = gam[ns]; S->ro = rom[ns]; S->beta = beta;
    s_bx[SYS_X] = beta * al;
    s_bx[SYS_YZ] = beta * al;
    s_bx[SYS_T] = 0.5 * al * dt / B.pec;     // SolveImpEqnUpdate_Temp.F90:25
  }
  __syncthreads();
  const int nx = B.nx, nxm = B.nxm;
  // row scale, sub- and super-diagonal (stored temporarily in C_FACT / C_DU)
  for (int t = threadIdx.x; t < 3 * nx; t += blockDim.x) {
    const int sys = t / nx, k = t % nx;
    double *sc = B.coef + (long long)(sys * C_N + C_SC) * nx;
    double *dl = B.coef + (long long)(sys * C_N + C_FACT) * nx;
    double *du = B.coef + (long long)(sys * C_N + C_DU) * nx;
    const double bx = s_bx[sys];
    double s = 1.0, am = 0.0, ap = 0.0;
    if (sys == SYS_X) {
      if (k >= 1 && k <= nxm - 1) {
        s = 1.0 / (1.0 - tabk(B, T_AC3CK, k) * bx);
        am = -tabk(B, T_AM3SSK, k) * bx * s;
        ap = -tabk(B, T_AP3SSK, k) * bx * s;
      }
    } else if (sys == SYS_YZ) {
      if (k <= nxm - 1) {
        s = 1.0 / (1.0 - tabk(B, T_AC3SK, k) * bx);
        am = -tabk(B, T_AM3SK, k) * bx * s;
        ap = -tabk(B, T_AP3SK, k) * bx * s;
      }
    } else {
      if (k >= 1 && k <= nxm - 1) {
        s = 1.0 / (1.0 - tabk(B, T_AC3SSK, k) * bx);
        am = -tabk(B, T_AM3SSK, k) * bx * s;
        ap = -tabk(B, T_AP3SSK, k) * bx * s;
      }
    }
    sc[k] = s; dl[k] = am; du[k] = ap;
  }
  __syncthreads();
  // sequential LU recurrence, one thread per system
  if (threadIdx.x < 3) {
    const int sys = threadIdx.x;
    const int n = (sys == SYS_YZ) ? nxm : nx;
    double *dl = B.coef + (long long)(sys * C_N + C_FACT) * nx;   // in: amkl, out: fact
    double *du = B.coef + (long long)(sys * C_N + C_DU) * nx;
    double *dp = B.coef + (long long)(sys * C_N + C_DP) * nx;
    double *g = B.coef + (long long)(sys * C_N + C_G) * nx;
    double d = 1.0;
    dp[0] = 1.0;
    double am_next = dl[1 < n ? 1 : 0];
    dl[0] = 0.0;
    double gk = 1.0;
    g[0] = 1.0;
    int pivot_needed = 0;
    for (int k = 0; k < n - 1; ++k) {
      const double am = am_next;                  // amkl(k+1), the subdiagonal of row k+1
      if (k + 2 < n) am_next = dl[k + 2];
      if (fabs(d) < fabs(am)) pivot_needed = 1;
      const double fact = am / d;                 // dgttrf: FACT = DL(I)/D(I)
      d = 1.0 - fact * du[k];                     //         D(I+1) = D(I+1) - FACT*DU(I)
      dl[k + 1] = fact;
      dp[k + 1] = d;
      gk = -fact * gk;
      g[k + 1] = gk;
    }
    for (int k = n; k < nx; ++k) { dl[k] = 0.0; dp[k] = 1.0; g[k] = 0.0; }
    if (pivot_needed) atomicExch(&S->status, -2);
  }
}

constexpr int K1_TJ = 32;                       // tile width along y (one warp)
constexpr int K1_HJ = K1_TJ + 2;
constexpr int K1_NTAB = 14;                     // per-k scalars staged per plane

// tile of 32 x TI columns (one warp per row of the tile), halo of one cell
template <int TI>
struct K1Shape {
  static constexpr int HI = TI + 2;
  static constexpr int PL = K1_HJ * HI;         // one halo plane of one field
  static constexpr int NT = K1_TJ * TI;         // threads per block
  static constexpr int NLD = (PL + NT - 1) / NT; // halo elements each thread copies
};

// per-k scalar slots staged in shared memory
enum K1Tab { KT_UDX3M = 0, KT_UDX3C, KT_AM3SK, KT_AC3SK, KT_AP3SK, KT_AM3CK, KT_AC3CK, KT_AP3CK,
             KT_XSC, KT_XF, KT_YSC, KT_YF, KT_TSC, KT_TF };

// Values of plane k-1 that the stencils at plane k read, kept in registers
// by the thread of the column (its own column, plus vy at j+1 and vz at i+1).
struct K1Prev {
  double vx, vy, vy_jp, vz, vz_ip, t, pr;
};

// Accessor over the ring (planes k and k+1, 1-cell halo) and the stash of
// plane k-1.  Every plane-(k-1) access of the stencil formulas is one of the
// seven stashed values.
template <int PL>
struct RingAcc {
  const double *ring;   // [slot][field][PL]
  int s_c, s_p;         // slots of k and k+1
  int off;              // (ti+1)*K1_HJ + tj+1
  K1Prev prev;
  __device__ __forceinline__ double operator()(int f, int dk, int dj, int di) const {
    if (dk < 0) {
      if (f == F_VX) return prev.vx;
      if (f == F_VY) return dj > 0 ? prev.vy_jp : prev.vy;
      if (f == F_VZ) return di > 0 ? prev.vz_ip : prev.vz;
      if (f == F_T) return prev.t;
      return prev.pr;
    }
    const int s = dk > 0 ? s_p : s_c;
    return ring[(s * F_NF + f) * PL + off + di * K1_HJ + dj];
  }
};


__device__ __forceinline__ const double *k1_tab_src(const BoxDev &B, int t, int k) {
  switch (t) {
    case KT_UDX3M: return B.tab + (long long)T_UDX3M * B.nx + k;
    case KT_UDX3C: return B.tab + (long long)T_UDX3C * B.nx + k;
    case KT_AM3SK: return B.tab + (long long)T_AM3SK * B.nx + k;
    case KT_AC3SK: return B.tab + (long long)T_AC3SK * B.nx + k;
    case KT_AP3SK: return B.tab + (long long)T_AP3SK * B.nx + k;
    case KT_AM3CK: return B.tab + (long long)T_AM3CK * B.nx + k;
    case KT_AC3CK: return B.tab + (long long)T_AC3CK * B.nx + k;
    case KT_AP3CK: return B.tab + (long long)T_AP3CK * B.nx + k;
    case KT_XSC: return B.coef + (long long)(SYS_X * C_N + C_SC) * B.nx + k;
    case KT_XF: return B.coef + (long long)(SYS_X * C_N + C_FACT) * B.nx + k;
    case KT_YSC: return B.coef + (long long)(SYS_YZ * C_N + C_SC) * B.nx + k;
    case KT_YF: return B.coef + (long long)(SYS_YZ * C_N + C_FACT) * B.nx + k;
    case KT_TSC: return B.coef + (long long)(SYS_T * C_N + C_SC) * B.nx + k;
    default: return B.coef + (long long)(SYS_T * C_N + C_FACT) * B.nx + k;
  }
}

// ---------------------------------------------------------------------------
// K1: explicit terms + implicit rhs + forward elimination for all four
// fields, one thread per (j, i) column marching k upwards, PPB planes per
// block barrier.  MINB is the occupancy target (resident blocks per SM; 3
// caps registers at 80, 2 at 128).  Shared memory holds a ring of x-planes
// of vx, vy, vz, temp, pr (tile plus a 1-cell halo) and of the per-k metric
// and LU scalars, fetched with cp.async 2 PPB + 1 planes ahead so that each
// load has two barrier intervals of compute to arrive in.  Plane k-1 is not
// read from the ring: the seven values of it that the stencils need are kept
// in registers.  The RK history (the tile's own columns of rux, ruy, ruz,
// rutemp) travels in the same ring as aligned 16-byte pairs, so no global
// load of the march is waited for in registers.  Global stores use the global
// state space explicitly (st.global intrinsics), so the compiler knows they
// cannot touch the shared ring and keeps stencil values in registers across
// them.  Writes the RK history (rux.. = H) and the
// forward-sweep values y of each solve; the temperature sweep starts from
// y(1) = 0 and the missing contribution of its wall row is added by K2 (the
// solve is linear in y(1)).
// ---------------------------------------------------------------------------
template <int PPB, int TI = 8>
struct K1Ring {
  static constexpr int D = 2 * PPB + 1;        // prefetch distance in planes
  static constexpr int NS = D + PPB;           // ring slots
  static constexpr int HS = 4 * K1Shape<TI>::NT; // RK history of one plane (tile interior, 4 fields)
  static constexpr int SMEM = (NS * F_NF * K1Shape<TI>::PL + NS * 16 + NS * HS) * 8;
};

template <int TI, int MINB, int PPB>
__global__ void __launch_bounds__(K1Shape<TI>::NT, MINB) k_explicit_implicit_fwd(BatchDev bt, int ns) {
  constexpr int NS = K1Ring<PPB, TI>::NS;
  constexpr int D = K1Ring<PPB, TI>::D;
  constexpr int PL = K1Shape<TI>::PL, NT = K1Shape<TI>::NT, NLD = K1Shape<TI>::NLD;
  constexpr int HS = K1Ring<PPB, TI>::HS;
  extern __shared__ double k1sm[];
  double *ring = k1sm;
  double *tring = k1sm + NS * F_NF * PL;         // [slot][16]
  double *hring = tring + NS * 16;               // [slot][field][NT], the column of thread t at t
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  const BoxScalars *S = B.sc;
  if (S->status != 0) return;
  const int tid = threadIdx.x;
  const int tile = blockIdx.x - __ldg(bt.tile_off + b);
  const int nym = B.nym, nzm = B.nzm;
  const int ntj = (nym + K1_TJ - 1) / K1_TJ;
  const int j0 = (tile % ntj) * K1_TJ;
  const int i0 = (tile / ntj) * TI;
  const int tj = tid % K1_TJ;
  const int ti = tid / K1_TJ;
  const int j = j0 + tj, i = i0 + ti;
  const bool inside = (j < nym) && (i < nzm);
  const long long P = B.plane;
  const long long col = (long long)i * nym + j;
  const int nx = B.nx, nxm = B.nxm;
  const StencilConst c = make_sconst(B);
  const double al = S->al, ga = S->ga, ro = S->ro, dt = S->dt;
  const double alre = al / B.ren;
  const double alpec = al / B.pec;
  const double udy_al = B.dy * al;
  const double dz_ = B.dz;

  const double *fld[F_NF] = {B.vx, B.vy, B.vz, B.temp, B.pr};

  // this thread's halo elements: r = tid + q NT for q < NLD while r < PL
  long long g[NLD];
#pragma unroll
  for (int q = 0; q < NLD; ++q) {
    const int r = tid + q * NT;
    const int hi = r / K1_HJ, hj = r - hi * K1_HJ;
    const int jj = (j0 + hj - 1 + nym) % nym, ii = (i0 + hi - 1 + nzm) % nzm;
    g[q] = (long long)ii * nym + jj;
  }
  // source of this thread's per-k scalar (threads tid < K1_NTAB), resolved
  // once: inside the march every descriptor read after a global store is a
  // reload, and the 14 cases would diverge within the first warp each plane
  const double *tsrc = tid < K1_NTAB ? k1_tab_src(B, tid, 0) : nullptr;
  // the RK history of a plane travels with it in the ring: 4 fields x NT
  // columns as 2 NT aligned 16-byte pairs, two per thread.  Pair r = tid +
  // q NT is field r / (NT/2), tile row c / 16 and columns 2 (c % 16) + {0, 1}
  // with c = r % (NT/2); a pair is inside the box or wholly outside it (j0
  // and nym are even)
  const double *hsrc[2];
  int hdst[2];
  bool hok[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int r = tid + q * NT, fq = r / (NT / 2), cc = r - fq * (NT / 2);
    const int hrow = cc / 16, hj = 2 * (cc % 16);
    const double *base = fq == 0 ? B.rux : fq == 1 ? B.ruy : fq == 2 ? B.ruz : B.rutemp;
    hok[q] = (i0 + hrow < nzm) && (j0 + hj < nym);
    hsrc[q] = base + (long long)(i0 + hrow) * nym + j0 + hj;
    hdst[q] = fq * NT + hrow * K1_TJ + hj;
  }
  auto load_plane = [&](int p) {      // plane p and its per-k scalars into slot p % NS
    if (p > nx - 1) return;
    const int sl = p % NS;
    double *dst = ring + sl * F_NF * PL;
    const long long po = (long long)p * P;
#pragma unroll
    for (int f = 0; f < F_NF; ++f) {
#pragma unroll
      for (int q = 0; q < NLD; ++q)
        if (q * NT + tid < PL) cp_async8(dst + f * PL + tid + q * NT, fld[f] + po + g[q]);
    }
    if (tid < K1_NTAB && p <= nxm - 1) cp_async8(tring + sl * 16 + tid, tsrc + p);
#pragma unroll
    for (int q = 0; q < 2; ++q)
      if (hok[q] && p <= nxm - 1) cp_async16(hring + sl * HS + hdst[q], hsrc[q] + (long long)p * P);
  };
  // this column's history and forward-sweep outputs, resolved once (read
  // from the descriptor inside the march, each would be reloaded after every
  // global store, which might alias the descriptor)
  double *const rux = B.rux + col, *const ruy = B.ruy + col, *const ruz = B.ruz + col, *const rut = B.rutemp + col;
  double *const yb0 = B.ybuf[0] + col, *const yb1 = B.ybuf[1] + col, *const yb2 = B.ybuf[2] + col,
                *const yb3 = B.ybuf[3] + col;

  RingAcc<PL> acc;
  acc.ring = ring;
  acc.off = (ti + 1) * K1_HJ + tj + 1;
  acc.prev = K1Prev{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};

  // forward-sweep carries
  double yX = inside ? B.wall[col] : 0.0;   // rhs(1,j,i) left by the last vz solve
  double yY = 0.0, yZ = 0.0, yT = 0.0;

  for (int p = 0; p < D - PPB; ++p) load_plane(p);
  cp_async_commit();
  for (int p = D - PPB; p < D; ++p) load_plane(p);
  cp_async_commit();
  cp_async_wait_1();
  __syncthreads();

  for (int k0 = 0; k0 < nxm; k0 += PPB) {
#pragma unroll
    for (int u = 0; u < PPB; ++u) load_plane(k0 + D + u);
    cp_async_commit();
#pragma unroll
    for (int u = 0; u < PPB; ++u) {
      const int kc = k0 + u;
      if (kc >= nxm) break;
      acc.s_c = kc % NS;
      acc.s_p = (kc + 1) % NS;
      const double *tk = tring + (kc % NS) * 16;
      const double *hk = hring + (kc % NS) * HS + tid;   // this column's history, field f at hk[f NT]
      if (inside) {
        const long long o = (long long)kc * P;
        const int dkm = kc == 0 ? 0 : -1;
        const int dkp = kc == nxm - 1 ? 0 : 1;
        const double udx3m_k = tk[KT_UDX3M];
        const double am_s = tk[KT_AM3SK], ac_s = tk[KT_AC3SK], ap_s = tk[KT_AP3SK];
        // vy, vz: rows kc = 0..nxm-1 of the size-nxm systems
        {
          const double H = h_vy(acc, c, udx3m_k, dkm, dkp);
          const double dyp = (acc(F_PR, 0, 0, 0) - acc(F_PR, 0, -1, 0)) * udy_al;
          const double r = rhs_vyz(H, hk[1 * NT], acc(F_VY, dkp, 0, 0), acc(F_VY, 0, 0, 0),
                                   acc(F_VY, dkm, 0, 0), am_s, ac_s, ap_s, dyp, ga, ro, alre, dt);
          __stwb(ruy + o, H);
          const double bb = r * tk[KT_YSC];
          yY = (kc == 0) ? bb : bb - tk[KT_YF] * yY;
          __stwb(yb1 + o, yY);
        }
        {
          const double H = h_vz(acc, c, udx3m_k, dkm, dkp);
          const double dzp = (acc(F_PR, 0, 0, 0) - acc(F_PR, 0, 0, -1)) * dz_ * al;
          const double r = rhs_vyz(H, hk[2 * NT], acc(F_VZ, dkp, 0, 0), acc(F_VZ, 0, 0, 0),
                                   acc(F_VZ, dkm, 0, 0), am_s, ac_s, ap_s, dzp, ga, ro, alre, dt);
          __stwb(ruz + o, H);
          const double bb = r * tk[KT_YSC];
          yZ = (kc == 0) ? bb : bb - tk[KT_YF] * yZ;
          __stwb(yb2 + o, yZ);
        }
        if (kc >= 1) {
          const double udx3c_k = tk[KT_UDX3C];
          const double am_c = tk[KT_AM3CK], ac_c = tk[KT_AC3CK], ap_c = tk[KT_AP3CK];
          {
            const double H = h_vx(acc, c, udx3c_k);
            const double r = rhs_vx(H, hk[0], acc(F_VX, 1, 0, 0), acc(F_VX, 0, 0, 0),
                                    acc(F_VX, -1, 0, 0), acc(F_PR, 0, 0, 0), acc(F_PR, -1, 0, 0),
                                    am_c, ac_c, ap_c, al, ga, ro, alre, dt, udx3c_k);
            __stwb(rux + o, H);
            const double bb = r * tk[KT_XSC];
            yX = bb - tk[KT_XF] * yX;
            __stwb(yb0 + o, yX);
          }
          {
            const double H = h_temp(acc, c, udx3c_k);
            const double r = rhs_temp(H, hk[3 * NT], acc(F_T, 1, 0, 0), acc(F_T, 0, 0, 0),
                                      acc(F_T, -1, 0, 0), am_c, ac_c, ap_c, ga, ro, alpec, dt);
            __stwb(rut + o, H);
            const double bb = r * tk[KT_TSC];
            yT = bb - tk[KT_TF] * yT;
            __stwb(yb3 + o, yT);
          }
        }
        // stash what plane kc+1 will need of this plane
        acc.prev.vx = acc(F_VX, 0, 0, 0);
        acc.prev.vy = acc(F_VY, 0, 0, 0);
        acc.prev.vy_jp = acc(F_VY, 0, 1, 0);
        acc.prev.vz = acc(F_VZ, 0, 0, 0);
        acc.prev.vz_ip = acc(F_VZ, 0, 0, 1);
        acc.prev.t = acc(F_T, 0, 0, 0);
        acc.prev.pr = acc(F_PR, 0, 0, 0);
      }
    }
    cp_async_wait_1();
    __syncthreads();
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// K2: backward substitution and update (SolveImpEqnUpdate_*: dgttrs back
// sweep, q += dq), then the wall conditions of ImplicitAndUpdateVX.F90:76-77
// and ImplicitAndUpdateTemp.F90:69-73.  One thread per column.
// ---------------------------------------------------------------------------
constexpr int K2_U = 3;   // planes loaded per chunk (loads of a chunk are all in flight together; 4 spills at 80 registers)

__global__ void __launch_bounds__(256, 3) k_implicit_bwd(BatchDev bt, int ns) {
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  if (B.sc->status != 0) return;
  const long long col = (long long)(blockIdx.x - __ldg(bt.tile_off + b)) * blockDim.x + threadIdx.x;
  if (col >= B.plane) return;
  const int nx = B.nx, nxm = B.nxm;
  const long long P = B.plane;
  // the LU rows of the three systems, as offsets from one base (seven
  // separate pointers would hold 14 registers across both sweeps)
  const double *__restrict__ cf = B.coef;
  const auto lu = [&](int sys, int arr, int k) { return __ldg(cf + (long long)(sys * C_N + arr) * nx + k); };
  const double *__restrict__ y0 = B.ybuf[0] + col;
  const double *__restrict__ y1 = B.ybuf[1] + col;
  const double *__restrict__ y2 = B.ybuf[2] + col;
  const double *__restrict__ y3 = B.ybuf[3] + col;
  double *__restrict__ vx = B.vx + col;
  double *__restrict__ vy = B.vy + col;
  double *__restrict__ vz = B.vz + col;
  double *__restrict__ tp = B.temp + col;
  double xX = 0.0, xY = 0.0, xZ = 0.0;
  // sweep 1: vx (rows nxm-1..1 of size nx), vy and vz (rows nxm-1..0 of size nxm)
  for (int k0 = nxm - 1; k0 >= 0; k0 -= K2_U) {
    double a0[K2_U], a1[K2_U], a2[K2_U], q0[K2_U], q1[K2_U], q2[K2_U];
#pragma unroll
    for (int u = 0; u < K2_U; ++u) {
      const int k = k0 - u;
      if (k >= 0) {
        const long long o = (long long)k * P;
        a1[u] = y1[o]; a2[u] = y2[o]; q1[u] = vy[o]; q2[u] = vz[o];
        if (k >= 1) { a0[u] = y0[o]; q0[u] = vx[o]; }
      }
    }
#pragma unroll
    for (int u = 0; u < K2_U; ++u) {
      const int k = k0 - u;
      if (k < 0) break;
      const long long o = (long long)k * P;
      const double dy_ = lu(SYS_YZ, C_DP, k);
      if (k == nxm - 1) {
        xY = a1[u] / dy_;
        xZ = a2[u] / dy_;
      } else {
        const double uu = lu(SYS_YZ, C_DU, k);
        xY = (a1[u] - uu * xY) / dy_;
        xZ = (a2[u] - uu * xZ) / dy_;
      }
      vy[o] = q1[u] + xY;
      vz[o] = q2[u] + xZ;
      if (k >= 1) {
        xX = (a0[u] - lu(SYS_X, C_DU, k) * xX) / lu(SYS_X, C_DP, k);
        vx[o] = q0[u] + xX;
      }
    }
  }
  vx[0] = 0.0;
  vx[(long long)(nx - 1) * P] = 0.0;
  const double w = xZ;            // rhs(1,j,i) after the vz solve
  B.wall[col] = w;
  // sweep 2: temperature, with the wall row's contribution g(k) * w
  double xT = 0.0;
  for (int k0 = nxm - 1; k0 >= 1; k0 -= K2_U) {
    double a3[K2_U], q3[K2_U];
#pragma unroll
    for (int u = 0; u < K2_U; ++u) {
      const int k = k0 - u;
      if (k >= 1) { const long long o = (long long)k * P; a3[u] = y3[o]; q3[u] = tp[o]; }
    }
#pragma unroll
    for (int u = 0; u < K2_U; ++u) {
      const int k = k0 - u;
      if (k < 1) break;
      const double y = a3[u] + lu(SYS_T, C_G, k) * w;
      xT = (y - lu(SYS_T, C_DU, k) * xT) / lu(SYS_T, C_DP, k);
      tp[(long long)k * P] = q3[u] + xT;
    }
  }
  tp[0] = B.tempbp;
  tp[(long long)(nx - 1) * P] = B.temptp;
}

// ---------------------------------------------------------------------------
// Projection: CorrectVelocity.F90:19-44 and CorrectPressure.F90:19-51 in one
// pass over the cells k = 1..nxm.  Thread per cell.
// ---------------------------------------------------------------------------
constexpr int KC_U = 4;   // planes per prefetch chunk

__global__ void __launch_bounds__(256) k_correct(BatchDev bt, int ns, int do_vel, int do_pr) {
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  const BoxScalars *S = B.sc;
  if (S->status != 0) return;
  const long long col = (long long)(blockIdx.x - __ldg(bt.tile_off + b)) * blockDim.x + threadIdx.x;
  const long long P = B.plane;
  if (col >= P) return;
  const int nym = B.nym, nzm = B.nzm, nxm = B.nxm;
  const int i = (int)(col / nym);
  const int j = (int)(col - (long long)i * nym);
  const int im = i == 0 ? nzm - 1 : i - 1, ip = i == nzm - 1 ? 0 : i + 1;
  const int jm = j == 0 ? nym - 1 : j - 1, jp = j == nym - 1 ? 0 : j + 1;
  const long long oim = (long long)im * nym + j - col, oip = (long long)ip * nym + j - col;
  const long long ojm = (long long)i * nym + jm - col, ojp = (long long)i * nym + jp - col;
  const double *__restrict__ phi = B.phi + col;
  double *__restrict__ vx = B.vx + col;
  double *__restrict__ vy = B.vy + col;
  double *__restrict__ vz = B.vz + col;
  double *__restrict__ pr = B.pr + col;
  const double al = S->al, dt = S->dt;
  const double udy = al * dt * B.dy;
  const double udz = al * dt * B.dz;
  const double be = al * S->beta;
  const double dzq = B.dzq, dyq = B.dyq;
  double fm = phi[0];          // phi(kmv(k)) for k = 0 is phi(0)
  double fc = fm;
  for (int k0 = 0; k0 < nxm; k0 += KC_U) {
    double fn[KC_U], fzp[KC_U], fzm[KC_U], fyp[KC_U], fym[KC_U];
    double qx[KC_U], qy[KC_U], qz[KC_U], qp[KC_U];
#pragma unroll
    for (int u = 0; u < KC_U; ++u) {
      const int k = k0 + u;
      if (k < nxm) {
        const long long o = (long long)k * P;
        const int kn = k + 1 < nxm ? k + 1 : k;     // kpv
        fn[u] = phi[(long long)kn * P];
        fzp[u] = phi[o + oip]; fzm[u] = phi[o + oim];
        fyp[u] = phi[o + ojp]; fym[u] = phi[o + ojm];
        if (do_vel) { qx[u] = vx[o]; qy[u] = vy[o]; qz[u] = vz[o]; }
        if (do_pr) qp[u] = pr[o];
      }
    }
#pragma unroll
    for (int u = 0; u < KC_U; ++u) {
      const int k = k0 + u;
      if (k >= nxm) break;
      const long long o = (long long)k * P;
      const double f = fc;
      if (do_vel) {
        // CorrectVelocity.F90:32-41
        const double usukm = al * dt * tabk(B, T_UDX3C, k);
        if (k >= 1) vx[o] = qx[u] - (f - fm) * usukm;
        vy[o] = qy[u] - (f - fym[u]) * udy;
        vz[o] = qz[u] - (f - fzm[u]) * udz;
      }
      if (do_pr) {
        // CorrectPressure.F90:33-48 (kpv/kmv clamp at the walls)
        const double amm = tabk(B, T_AMPHK, k), acc = tabk(B, T_ACPHK, k), app = tabk(B, T_APPHK, k);
        const double fkm = k == 0 ? f : fm;
        const double zz = (fzp[u] - 2.0 * f + fzm[u]) * dzq;
        const double yy = (fyp[u] - 2.0 * f + fym[u]) * dyq;
        const double xx = fn[u] * app + f * acc + fkm * amm;
        pr[o] = qp[u] + f - be * (zz + yy + xx);
      }
      fm = f;
      fc = fn[u];
    }
  }
}

// ---------------------------------------------------------------------------
// Divergence into the phi buffer (CalcLocalDivergence.F90:20-40); used by the
// routine-level entry point (the fused path computes it inside the y-FFT).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double local_div(const BoxDev &B, int k, int j, int i) {
  const long long P = B.plane;
  const int nym = B.nym, nzm = B.nzm;
  const int ip = i == nzm - 1 ? 0 : i + 1;
  const int jp = j == nym - 1 ? 0 : j + 1;
  const long long o = (long long)k * P + (long long)i * nym + j;
  return (B.vz[(long long)k * P + (long long)ip * nym + j] - B.vz[o]) * B.dz
       + (B.vy[(long long)k * P + (long long)i * nym + jp] - B.vy[o]) * B.dy
       + (B.vx[o + P] - B.vx[o]) * tabk(B, T_UDX3M, k);
}

// Column march: one thread per (j, i), planes in chunks whose loads are all
// in flight together; vx(k+1) of one plane is vx(k) of the next.
constexpr int KD_U = 4;
__global__ void __launch_bounds__(256, 2) k_divergence(BatchDev bt, int ns) {
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active || ns >= B.nsst) return;
  const BoxScalars *S = B.sc;
  if (S->status != 0) return;
  const long long col = (long long)(blockIdx.x - __ldg(bt.tile_off + b)) * blockDim.x + threadIdx.x;
  const long long P = B.plane;
  if (col >= P) return;
  const int nym = B.nym, nzm = B.nzm, nxm = B.nxm;
  const int i = (int)(col / nym);
  const int j = (int)(col - (long long)i * nym);
  const long long oip = (long long)(i == nzm - 1 ? 0 : i + 1) * nym + j - col;
  const long long ojp = (long long)i * nym + (j == nym - 1 ? 0 : j + 1) - col;
  const double *__restrict__ vx = B.vx + col;
  const double *__restrict__ vy = B.vy + col;
  const double *__restrict__ vz = B.vz + col;
  double *__restrict__ phi = B.phi + col;
  const double usdtal = 1.0 / (S->dt * S->al);
  const double dz = B.dz, dy = B.dy;
  const double *__restrict__ t_udx3m = B.tab + (long long)T_UDX3M * B.nx;   // resolved before the stores
  double xk = vx[0];
  for (int k0 = 0; k0 < nxm; k0 += KD_U) {
    double zc[KD_U], zp[KD_U], yc[KD_U], yp[KD_U], xn[KD_U];
#pragma unroll
    for (int u = 0; u < KD_U; ++u) {
      const int k = k0 + u;
      if (k < nxm) {
        const long long o = (long long)k * P;
        zc[u] = vz[o]; zp[u] = vz[o + oip];
        yc[u] = vy[o]; yp[u] = vy[o + ojp];
        xn[u] = vx[o + P];
      }
    }
#pragma unroll
    for (int u = 0; u < KD_U; ++u) {
      const int k = k0 + u;
      if (k >= nxm) break;
      // CalcLocalDivergence.F90:34-37
      const double dq = (zp[u] - zc[u]) * dz + (yp[u] - yc[u]) * dy + (xn[u] - xk) * __ldg(t_udx3m + k);
      phi[(long long)k * P] = dq * usdtal;
      xk = xn[u];
    }
  }
}

// ---------------------------------------------------------------------------
// Diagnostics over the current velocity: CFL (CalcMaxCFL.F90:29-39), max
// |div| (CheckDivergence.F90:29-38) and vmax (GlobalQuantities.F90:44-46).
// Block max + atomicMax on the bit pattern (values are >= 0).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Column march as in k_divergence: one thread per (j, i); vx(k+1) of one
// plane is vx(k) of the next, so every field is read once.  In a step
// (every_box = 0) a failed or held box is skipped; the routine-level calls
// (CalcMaxCFL, CheckDivergence) evaluate the box whatever its status.
__global__ void __launch_bounds__(256, 2) k_diag(BatchDev bt, int every_box) {
  const int b = find_box(bt.tile_off, bt.nbox, blockIdx.x);
  const BoxDev &B = bt.boxes[b];
  if (!B.active) return;
  BoxScalars *S = B.sc;
  if (!every_box && S->status != 0) return;
  const long long P = B.plane;
  const long long col = (long long)(blockIdx.x - __ldg(bt.tile_off + b)) * blockDim.x + threadIdx.x;
  double cfl = 0.0, dv = 0.0, my = 0.0, mz = 0.0;
  int bad = 0;
  if (col < P) {
    const int nym = B.nym, nzm = B.nzm, nxm = B.nxm;
    const int i = (int)(col / nym);
    const int j = (int)(col - (long long)i * nym);
    const long long oip = (long long)(i == nzm - 1 ? 0 : i + 1) * nym + j - col;
    const long long ojp = (long long)i * nym + (j == nym - 1 ? 0 : j + 1) - col;
    const double *__restrict__ vx = B.vx + col;
    const double *__restrict__ vy = B.vy + col;
    const double *__restrict__ vz = B.vz + col;
    const double *__restrict__ tp = B.temp + col;
    const double dz = B.dz, dy = B.dy;
    double xk = vx[0];
    for (int k0 = 0; k0 < nxm; k0 += KD_U) {
      double zc[KD_U], zp[KD_U], yc[KD_U], yp[KD_U], xn[KD_U], tc[KD_U];
#pragma unroll
      for (int u = 0; u < KD_U; ++u) {
        const int k = k0 + u;
        if (k < nxm) {
          const long long o = (long long)k * P;
          zc[u] = vz[o]; zp[u] = vz[o + oip];
          yc[u] = vy[o]; yp[u] = vy[o + ojp];
          xn[u] = vx[o + P];
          tc[u] = tp[o];
        }
      }
#pragma unroll
      for (int u = 0; u < KD_U; ++u) {
        const int k = k0 + u;
        if (k >= nxm) break;
        const double udx3m = tabk(B, T_UDX3M, k);
        const double q = fabs((zc[u] + zp[u]) * 0.5 * dz) + fabs((yc[u] + yp[u]) * 0.5 * dy)
                       + fabs((xk + xn[u]) * 0.5 * udx3m);
        const double d = (zp[u] - zc[u]) * dz + (yp[u] - yc[u]) * dy + (xn[u] - xk) * udx3m;
        if (!isfinite(q) || !isfinite(d) || !isfinite(tc[u])) bad = 1;
        cfl = fmax(cfl, q);
        dv = fmax(dv, fabs(d));
        my = fmax(my, fabs(yc[u]));
        mz = fmax(mz, fabs(zc[u]));
        xk = xn[u];
      }
    }
  }
  cfl = warp_max(cfl); dv = warp_max(dv); my = warp_max(my); mz = warp_max(mz);
  __shared__ double sm[4][8];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sm[0][w] = cfl; sm[1][w] = dv; sm[2][w] = my; sm[3][w] = mz; }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(&S->nonfinite, 1);
  if (threadIdx.x < 4) {
    double m = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) m = fmax(m, sm[threadIdx.x][q]);
    atomicMax(&S->red_u64[threadIdx.x], dbits(m));
  }
}

// Plate Nusselt numbers (CalcPlateNu.F90:24-43): per-block partial sums, in a
// fixed number of blocks per box so that the final sum order is fixed.
constexpr int NU_BLOCKS = 32;
__global__ void __launch_bounds__(256) k_plate_nu(const BoxDev *__restrict__ boxes, int nbox) {
  const int b = blockIdx.y;
  if (b >= nbox) return;
  const BoxDev &B = boxes[b];
  if (!B.active) return;
  const long long P = B.plane;
  const int nx = B.nx, nxm = B.nxm;
  const double del = 1.0 / (tabk(B, T_XC, 1) - tabk(B, T_XC, 0));
  const double deln = 1.0 / (tabk(B, T_XC, nx - 1) - tabk(B, T_XC, nxm - 1));
  double lo = 0.0, up = 0.0;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < P; c += (long long)NU_BLOCKS * blockDim.x) {
    lo += (B.temp[c] - B.temp[P + c]) * del;
    up += (B.temp[(long long)(nxm - 1) * P + c] - B.temp[(long long)(nx - 1) * P + c]) * deln;
  }
  __shared__ double s_lo[256], s_up[256];
  s_lo[threadIdx.x] = lo; s_up[threadIdx.x] = up;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) { s_lo[threadIdx.x] += s_lo[threadIdx.x + st]; s_up[threadIdx.x] += s_up[threadIdx.x + st]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { B.nu_part[2 * blockIdx.x] = s_lo[0]; B.nu_part[2 * blockIdx.x + 1] = s_up[0]; }
}

// ---------------------------------------------------------------------------
// Output-time diagnostics: per-plane horizontal sums and extrema of
// GlobalQuantities.F90:38-61, CalcStats (StatRoutines.F90:21-43) and
// CalcDissipationNu.F90:53-105, all in one pass over vx, vy, vz, temp.
// Block (c, k) reduces chunk c of the columns of plane k (k = 0..nxm-1,
// reading plane k+1 and the j+1, i+1 neighbours); the host adds the chunks
// of a plane in a fixed order and weights the planes.
// ---------------------------------------------------------------------------
enum PlaneQ {
  PQ_VX, PQ_VY, PQ_VZ, PQ_T, PQ_VX2, PQ_VY2, PQ_VZ2, PQ_T2, PQ_TVX,  // CalcStats
  PQ_TCVXC, PQ_TC,                                                  // GlobalQuantities
  PQ_DISSTE, PQ_DISSTE2, PQ_DISSTH,                                 // CalcDissipationNu
  PQ_NSUM,                                                          // sums above, maxima below
  PQ_MAXVZ = PQ_NSUM, PQ_MAXVY, PQ_MAXVX, PQ_MAXT, PQ_NEGMINT, PQ_N
};
constexpr int PS_CHUNKS = 16;

__global__ void __launch_bounds__(256) k_plane_sums(const BoxDev *__restrict__ bp, double *__restrict__ out) {
  const BoxDev &B = *bp;
  const int k = blockIdx.y, c = blockIdx.x;
  const int nym = B.nym, nzm = B.nzm, nxm = B.nxm;
  const long long P = B.plane;
  const double *xc = B.tab + (long long)T_XC * B.nx;
  // CalcDissipationNu.F90:32-40: dxc(k), and dxm(k) with the last plane
  // reusing the spacing of the cell centres below it
  const double dxc = 1.0 / (xc[k + 1] - xc[k]);
  const int km = k < nxm - 1 ? k : nxm - 2;
  const double dxm = 1.0 / ((xc[km + 1] + xc[km + 2]) * 0.5 - (xc[km] + xc[km + 1]) * 0.5);
  const double dy = B.dy, dz = B.dz;
  double s[PQ_N];
#pragma unroll
  for (int q = 0; q < PQ_N; ++q) s[q] = 0.0;
  s[PQ_MAXT] = -1.7976931348623157e308;
  s[PQ_NEGMINT] = -1.7976931348623157e308;
  const double *vx = B.vx + (long long)k * P, *vy = B.vy + (long long)k * P;
  const double *vz = B.vz + (long long)k * P, *tp = B.temp + (long long)k * P;
  for (long long col = (long long)c * blockDim.x + threadIdx.x; col < P; col += (long long)PS_CHUNKS * blockDim.x) {
    const int i = (int)(col / nym), j = (int)(col - (long long)i * nym);
    const long long oj = (long long)i * nym + (j == nym - 1 ? 0 : j + 1);
    const long long oi = (long long)(i == nzm - 1 ? 0 : i + 1) * nym + j;
    const double vx0 = vx[col], vx1 = vx[col + P], vxj = vx[oj], vxi = vx[oi];
    const double vy0 = vy[col], vy1 = vy[col + P], vyj = vy[oj], vyi = vy[oi];
    const double vz0 = vz[col], vz1 = vz[col + P], vzj = vz[oj], vzi = vz[oi];
    const double t0 = tp[col], t1 = tp[col + P], tj = tp[oj], ti = tp[oi];
    s[PQ_VX] += vx0; s[PQ_VY] += vy0; s[PQ_VZ] += vz0; s[PQ_T] += t0;
    s[PQ_VX2] += vx0 * vx0; s[PQ_VY2] += vy0 * vy0; s[PQ_VZ2] += vz0 * vz0; s[PQ_T2] += t0 * t0;
    s[PQ_TVX] += t0 * vx0;
    const double vxcen = (vx0 + vx1) * 0.5, tempcen = (t0 + t1) * 0.5;
    s[PQ_TCVXC] += tempcen * vxcen;
    s[PQ_TC] += tempcen;
    const double hxx = (vx1 - vx0) * dxc, hxy = (vxj - vx0) * dy, hxz = (vxi - vx0) * dz;
    const double hyx = (vy1 - vy0) * dxm, hyy = (vyj - vy0) * dy, hyz = (vyi - vy0) * dz;
    const double hzx = (vz1 - vz0) * dxm, hzy = (vzj - vz0) * dy, hzz = (vzi - vz0) * dz;
    s[PQ_DISSTE] += hxx * hxx + hxy * hxy + hxz * hxz;
    s[PQ_DISSTE2] += (hyx * hyx + hyy * hyy + hyz * hyz) + (hzx * hzx + hzy * hzy + hzz * hzz);
    const double tx = (t1 - t0) * dxc, ty = (tj - t0) * dy, tz = (ti - t0) * dz;
    s[PQ_DISSTH] += tx * tx + ty * ty + tz * tz;
    s[PQ_MAXVZ] = fmax(s[PQ_MAXVZ], fabs(vz0));
    s[PQ_MAXVY] = fmax(s[PQ_MAXVY], fabs(vy0));
    s[PQ_MAXVX] = fmax(s[PQ_MAXVX], fabs(vx0));
    s[PQ_MAXT] = fmax(s[PQ_MAXT], t0);
    s[PQ_NEGMINT] = fmax(s[PQ_NEGMINT], -t0);
  }
  __shared__ double red[8][PQ_N];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < PQ_N; ++q) {
    double v = s[q];
    for (int o = 16; o > 0; o >>= 1) {
      const double u = __shfl_xor_sync(0xffffffffu, v, o);
      v = q < PQ_NSUM ? v + u : fmax(v, u);
    }
    if (l == 0) red[w][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < PQ_N) {
    const int q = threadIdx.x;
    double v = red[0][q];
    for (int x = 1; x < (int)(blockDim.x >> 5); ++x) v = q < PQ_NSUM ? v + red[x][q] : fmax(v, red[x][q]);
    out[((long long)k * PS_CHUNKS + c) * PQ_N + q] = v;
  }
}

// Horizontal slabs of SlabDumper (SlabDumpRoutines.F90:15-24): for slab m
// at plane kslab[m] (0-based), (vx(k) + vx(k+1)) / 2, vy(k), vz(k), temp(k)
// into out[m][4][plane].
struct SlabList {
  int k[16];
};
__global__ void k_slab_gather(const BoxDev *__restrict__ bp, SlabList sl, int nslab, double *__restrict__ out) {
  const BoxDev &B = *bp;
  const long long P = B.plane;
  const int m = blockIdx.y;
  if (m >= nslab) return;
  const long long o = (long long)sl.k[m] * P;
  double *dst = out + (long long)m * 4 * P;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < P; c += (long long)gridDim.x * blockDim.x) {
    dst[c] = (B.vx[o + c] + B.vx[o + P + c]) * 0.5;
    dst[P + c] = B.vy[o + c];
    dst[2 * P + c] = B.vz[o + c];
    dst[3 * P + c] = B.temp[o + c];
  }
}

// Finalise the reductions of one box (thread per box): diagnostics, plate Nu
// and the reference's error codes.
//   mode 0: step start  -> cfl/div/vmax from k_diag, then the dt rule of
//           main.F90:171-189 (codes 165, 166)
//   mode 1: step end    -> time += dt, ntime += 1, plate Nu, velocity limit
//           (266, main.F90:204) and non-finite values (266)
__global__ void k_finalize(const BoxDev *__restrict__ boxes, int nbox, int mode) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbox) return;
  const BoxDev &B = boxes[b];
  if (!B.active) return;
  BoxScalars *S = B.sc;
  if (mode == 0) {
    if (S->status != 0) return;
    double cfl = __longlong_as_double((long long)S->red_u64[0]);
    S->divmax = __longlong_as_double((long long)S->red_u64[1]);
    S->vmax[1] = __longlong_as_double((long long)S->red_u64[2]);
    S->vmax[0] = __longlong_as_double((long long)S->red_u64[3]);
    for (int q = 0; q < 4; ++q) S->red_u64[q] = 0ull;
    cfl = fmax(cfl, 0.00000001);             // CalcMaxCFL.F90:21
    S->cfl = cfl;
    if (S->nonfinite) { S->status = 266; return; }
    // velocity limit (main.F90:204) and mass conservation (main.F90:220)
    if (S->vmax[0] > S->limitvel && S->vmax[1] > S->limitvel) { S->status = 266; return; }
    if (S->ntime >= 1 && S->resid > 0.0 && S->divmax > S->resid) { S->status = 169; return; }
    double dt = S->dt;
    if (S->idtv) {
      if (S->ntime > 1) {
        dt = (cfl < 1.0e-8) ? S->dtmax : S->cflmax / cfl;
        if (dt > S->dtmax) dt = S->dtmax;
      } else {
        dt = S->dtmin;
      }
      S->dt = dt;
      S->cfl_used = cfl;
      if (dt < S->dtmin) S->status = 166;
    } else {
      S->cfl_used = cfl * dt;
      if (S->cfl_used > S->cflmax) S->status = 165;
    }
  } else {
    if (S->status != 0) return;
    S->time += S->dt;
    S->ntime += 1;
    double lo = 0.0, up = 0.0;
    for (int q = 0; q < NU_BLOCKS; ++q) { lo += B.nu_part[2 * q]; up += B.nu_part[2 * q + 1]; }
    S->nu_bot = lo / (double)(B.nzm * B.nym);
    S->nu_top = up / (double)(B.nzm * B.nym);
    if (!isfinite(S->nu_bot) || !isfinite(S->nu_top)) S->status = 266;
    if (B.hist_cap > 0) {
      double *h = B.hist + (long long)((S->ntime - 1) % B.hist_cap) * HIST_FIELDS;
      h[0] = S->time; h[1] = S->dt; h[2] = S->cfl_used; h[3] = S->divmax;
      h[4] = S->nu_bot; h[5] = S->nu_top; h[6] = S->vmax[1]; h[7] = S->vmax[0];
    }
    // hold at the stop step or at an output time: main.F90's loop index is
    // ntime - 1 here, so its "ntime.eq.1" is the second step
    if (S->status == 0) {
      bool hold = S->stop_ntime > 0 && S->ntime >= S->stop_ntime;
      if (S->tout > 0.0 && (S->ntime == 2 || fmod(S->time, S->tout) < S->dt)) hold = true;
      if (S->tmax > 0.0 && S->time > S->tmax) hold = true;
      if (hold) S->status = AFID_STATUS_HELD_DEV;
    }
  }
}

// Release the boxes on hold among the listed ones (afid_box_resume).
__global__ void k_resume(const BoxDev *__restrict__ boxes, int nbox) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbox) return;
  BoxScalars *S = boxes[b].sc;
  if (S->status == AFID_STATUS_HELD_DEV) S->status = 0;
}

// ---------------------------------------------------------------------------
// Layout conversion between the reference's Fortran order q(k, j, i) (k
// fastest, nk rows) and the device order q[k][i][j].  32x32 smem tiles over
// (k, j) for each i.
// ---------------------------------------------------------------------------
__global__ void k_fortran_to_dev(const double *__restrict__ src, double *__restrict__ dst,
                                 int nk, int nym, int nzm, int ld_k) {
  __shared__ double t[32][33];
  const int i = blockIdx.z;
  const int k0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, k = k0 + threadIdx.x;
    if (j < nym && k < nk) t[r][threadIdx.x] = src[(long long)i * nym * ld_k + (long long)j * ld_k + k];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, j = j0 + threadIdx.x;
    if (j < nym && k < nk) dst[(long long)k * nym * nzm + (long long)i * nym + j] = t[threadIdx.x][r];
  }
}

__global__ void k_dev_to_fortran(const double *__restrict__ src, double *__restrict__ dst,
                                 int nk, int nym, int nzm, int ld_k) {
  __shared__ double t[32][33];
  const int i = blockIdx.z;
  const int k0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, j = j0 + threadIdx.x;
    if (j < nym && k < nk) t[r][threadIdx.x] = src[(long long)k * nym * nzm + (long long)i * nym + j];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, k = k0 + threadIdx.x;
    if (j < nym && k < nk) dst[(long long)i * nym * ld_k + (long long)j * ld_k + k] = t[threadIdx.x][r];
  }
}

}  // namespace afid
