// Routine-level kernels: one kernel per reference subroutine, used by the
// entry points that keep the reference's subroutine boundaries
// (afid_explicit_terms_*, afid_implicit_and_update_*).  They share the
// stencil formulas of k_stencil.cuh, read their neighbours straight from
// global memory and materialise the reference's module arrays (qcap, dph,
// dq, hro, rhs) instead of keeping them on chip.
#pragma once
#include "k_stencil.cuh"

namespace afid {

struct GlobAcc {
  const double *f[F_NF];
  long long P;
  int nym, nzm, k, j, i;
  __device__ __forceinline__ double operator()(int fi, int dk, int dj, int di) const {
    int jj = j + dj; jj = jj < 0 ? jj + nym : (jj >= nym ? jj - nym : jj);
    int ii = i + di; ii = ii < 0 ? ii + nzm : (ii >= nzm ? ii - nzm : ii);
    return f[fi][(long long)(k + dk) * P + (long long)ii * nym + jj];
  }
};

__device__ __forceinline__ GlobAcc make_gacc(const BoxDev &B, int k, int j, int i) {
  GlobAcc a;
  a.f[F_VX] = B.vx; a.f[F_VY] = B.vy; a.f[F_VZ] = B.vz; a.f[F_T] = B.temp; a.f[F_PR] = B.pr;
  a.P = B.plane; a.nym = B.nym; a.nzm = B.nzm; a.k = k; a.j = j; a.i = i;
  return a;
}

// ExplicitTerms{VX,VY,VZ,Temp}: H of one field for every cell of its range.
// field: 0 vx -> qcap (k=2..nxm), 1 vy -> dph (1..nxm), 2 vz -> dq (1..nxm),
// 3 temp -> hro (2..nxm).  Thread per (k, j, i) with k < nxm.
__global__ void __launch_bounds__(256) k_explicit_one(const BoxDev *__restrict__ boxes, int field) {
  const BoxDev &B = boxes[0];
  const long long P = B.plane;
  const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= (long long)B.nxm * P) return;
  const int k = (int)(cell / P);
  const long long col = cell - (long long)k * P;
  const int i = (int)(col / B.nym);
  const int j = (int)(col - (long long)i * B.nym);
  const StencilConst c = make_sconst(B);
  const GlobAcc a = make_gacc(B, k, j, i);
  const int dkm = k == 0 ? 0 : -1;
  const int dkp = k == B.nxm - 1 ? 0 : 1;
  if (field == F_VX) {
    if (k >= 1) B.qcap[cell] = h_vx(a, c, tabk(B, T_UDX3C, k));
  } else if (field == F_VY) {
    B.phi[cell] = h_vy(a, c, tabk(B, T_UDX3M, k), dkm, dkp);
  } else if (field == F_VZ) {
    B.dq[cell] = h_vz(a, c, tabk(B, T_UDX3M, k), dkm, dkp);
  } else {
    if (k >= 1) B.hro[cell] = h_temp(a, c, tabk(B, T_UDX3C, k));
  }
}

// ImplicitAndUpdate{VX,VY,VZ,Temp} + SolveImpEqnUpdate_{X,YZ,Temp}: rhs,
// history update, forward elimination into the rhs buffer, back substitution
// and q += dq, with the wall rows of the size-nx systems taken from / left in
// the carried rhs(1,:,:) plane exactly as the reference's shared rhs array
// does.  Thread per (j, i) column.
__global__ void __launch_bounds__(256) k_implicit_one(const BoxDev *__restrict__ boxes, int field) {
  const BoxDev &B = boxes[0];
  const BoxScalars *S = B.sc;
  const long long P = B.plane;
  const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= P) return;
  const int i = (int)(col / B.nym);
  const int j = (int)(col - (long long)i * B.nym);
  const int nx = B.nx, nxm = B.nxm;
  const double al = S->al, ga = S->ga, ro = S->ro, dt = S->dt;
  const double alre = al / B.ren, alpec = al / B.pec;
  const int sys = field == F_VX ? SYS_X : (field == F_T ? SYS_T : SYS_YZ);
  const double *csc = coefp(B, sys, C_SC), *cf = coefp(B, sys, C_FACT);
  const double *cdp = coefp(B, sys, C_DP), *cdu = coefp(B, sys, C_DU);
  double *rhs = B.rhs;
  const int k0 = (field == F_VX || field == F_T) ? 1 : 0;
  const int n = (sys == SYS_YZ) ? nxm : nx;
  // forward elimination (rhs scaled by the row factor, then dgttrs forward)
  double y = (sys == SYS_YZ) ? 0.0 : B.wall[col];
  for (int k = k0; k < nxm; ++k) {
    const long long o = (long long)k * P + col;
    const GlobAcc a = make_gacc(B, k, j, i);
    double r;
    if (field == F_VX) {
      const double H = B.qcap[o];
      r = rhs_vx(H, B.rux[o], a(F_VX, 1, 0, 0), a(F_VX, 0, 0, 0), a(F_VX, -1, 0, 0),
                 a(F_PR, 0, 0, 0), a(F_PR, -1, 0, 0),
                 tabk(B, T_AM3CK, k), tabk(B, T_AC3CK, k), tabk(B, T_AP3CK, k),
                 al, ga, ro, alre, dt, tabk(B, T_UDX3C, k));
      B.rux[o] = H;
    } else if (field == F_VY || field == F_VZ) {
      const int dkm = k == 0 ? 0 : -1;
      const int dkp = k == nxm - 1 ? 0 : 1;
      const int fq = field;
      double dp;
      double H, Hold;
      if (field == F_VY) {
        dp = (a(F_PR, 0, 0, 0) - a(F_PR, 0, -1, 0)) * (B.dy * al);
        H = B.phi[o]; Hold = B.ruy[o];
        B.ruy[o] = H;
      } else {
        dp = (a(F_PR, 0, 0, 0) - a(F_PR, 0, 0, -1)) * B.dz * al;
        H = B.dq[o]; Hold = B.ruz[o];
        B.ruz[o] = H;
      }
      r = rhs_vyz(H, Hold, a(fq, dkp, 0, 0), a(fq, 0, 0, 0), a(fq, dkm, 0, 0),
                  tabk(B, T_AM3SK, k), tabk(B, T_AC3SK, k), tabk(B, T_AP3SK, k),
                  dp, ga, ro, alre, dt);
    } else {
      const double H = B.hro[o];
      r = rhs_temp(H, B.rutemp[o], a(F_T, 1, 0, 0), a(F_T, 0, 0, 0), a(F_T, -1, 0, 0),
                   tabk(B, T_AM3CK, k), tabk(B, T_AC3CK, k), tabk(B, T_AP3CK, k),
                   ga, ro, alpec, dt);
      B.rutemp[o] = H;
    }
    const double bb = r * __ldg(csc + k);
    y = (k == 0) ? bb : bb - __ldg(cf + k) * y;
    rhs[o] = y;
  }
  // back substitution (row nx of the size-nx systems holds rhs(nx) = 0)
  double x = 0.0;
  double *q = field == F_VX ? B.vx : field == F_VY ? B.vy : field == F_VZ ? B.vz : B.temp;
  for (int k = nxm - 1; k >= k0; --k) {
    const long long o = (long long)k * P + col;
    if (sys == SYS_YZ && k == nxm - 1) x = rhs[o] / __ldg(cdp + k);
    else x = (rhs[o] - __ldg(cdu + k) * x) / __ldg(cdp + k);
    q[o] = q[o] + x;
  }
  (void)n;
  if (sys == SYS_YZ) {
    B.wall[col] = x;                  // rhs(1,j,i) now holds dq(1)
  } else if (field == F_VX) {
    B.vx[col] = 0.0;
    B.vx[(long long)(nx - 1) * P + col] = 0.0;
  } else {
    B.temp[col] = B.tempbp;
    B.temp[(long long)(nx - 1) * P + col] = B.temptp;
  }
}

// ---------------------------------------------------------------------------
// Restart onto a new grid (ReadFlowField.F90:63-150, interp.F90:11-227): one
// thread per point of the new grid, written in the device layout.  The old
// field a(1:nxo, 1:nyom, 1:nzom) is the continua dataset in Fortran order;
// its halo is extrapolated on the fly as interp.F90:95-117 fills it, on the
// six faces only (edges and corners, which the reference never writes, are
// zero).  ``tab`` holds per new point of each direction (z: nzm, then y: nym,
// then x: nx entries) the new coordinate, the two bracketing old
// coordinates and their indices (interp.F90:128-175), each as a row of the
// direction's length.  The stencil and the operation order are those of
// interp.F90:177-227 and interptrilin, including the three upper-x corners
// read at the lower x index (sffc, sccc, scfc).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double interp_old(const double *__restrict__ a, int nxo, int nyom, int nzom,
                                             int k, int j, int i) {
  const int hx = (k == 0 || k == nxo + 1), hy = (j == 0 || j == nyom + 1), hz = (i == 0 || i == nzom + 1);
  const auto A = [&](int kk, int jj, int ii) {
    return __ldg(a + (kk - 1) + (long long)nxo * ((jj - 1) + (long long)nyom * (ii - 1)));
  };
  if (hx + hy + hz == 0) return A(k, j, i);
  if (hx + hy + hz > 1) return 0.0;
  if (hx) return k == 0 ? 2.0 * A(1, j, i) - A(2, j, i) : 2.0 * A(nxo, j, i) - A(nxo - 1, j, i);
  if (hz) return i == 0 ? 2.0 * A(k, j, 1) - A(k, j, 2) : 2.0 * A(k, j, nzom) - A(k, j, nzom - 1);
  return j == 0 ? 2.0 * A(k, 1, i) - A(k, 2, i) : 2.0 * A(k, nyom, i) - A(k, nyom - 1, i);
}

__global__ void __launch_bounds__(256) k_interp(const double *__restrict__ a, int nxo, int nyom, int nzom,
                                                const double *__restrict__ tab, double *__restrict__ out,
                                                int nx, int nym, int nzm) {
  const long long plane = (long long)nym * nzm;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)nx * plane) return;
  const int k = (int)(q / plane);
  const long long r = q - (long long)k * plane;
  const int i = (int)(r / nym), j = (int)(r - (long long)i * nym);
  const double *tx = tab, *ty = tab + 5LL * nzm, *tz = ty + 5LL * nym;
  const double bix = tx[i], bix1 = tx[nzm + i], bix2 = tx[2 * nzm + i];
  const int fi = (int)tx[3 * nzm + i], ci = (int)tx[4 * nzm + i];
  const double biy = ty[j], biy1 = ty[nym + j], biy2 = ty[2 * nym + j];
  const int fj = (int)ty[3 * nym + j], cj = (int)ty[4 * nym + j];
  const double biz = tz[k], biz1 = tz[nx + k], biz2 = tz[2 * nx + k];
  const int fk = (int)tz[3 * nx + k], ck = (int)tz[4 * nx + k];
  const double aficjfk = interp_old(a, nxo, nyom, nzom, fk, cj, fi);
  const double afifjfk = interp_old(a, nxo, nyom, nzom, fk, fj, fi);
  const double acicjfk = interp_old(a, nxo, nyom, nzom, fk, cj, ci);
  const double acifjfk = interp_old(a, nxo, nyom, nzom, fk, fj, ci);
  const double aficjck = interp_old(a, nxo, nyom, nzom, ck, cj, fi);
  const double afifjck = afifjfk;   // sffc = arrold(bifk, bifj, bifi)
  const double acicjck = acicjfk;   // sccc = arrold(bifk, bicj, bici)
  const double acifjck = acifjfk;   // scfc = arrold(bifk, bifj, bici)
  const double dxdydz = 1.0 / ((bix2 - bix1) * (biy2 - biy1) * (biz2 - biz1));
  out[q] = (aficjfk * (bix2 - bix) * (biy - biy1) * (biz2 - biz)
            + afifjfk * (bix2 - bix) * (biy2 - biy) * (biz2 - biz)
            + acicjfk * (bix - bix1) * (biy - biy1) * (biz2 - biz)
            + acifjfk * (bix - bix1) * (biy2 - biy) * (biz2 - biz)
            + aficjck * (bix2 - bix) * (biy - biy1) * (biz - biz1)
            + afifjck * (bix2 - bix) * (biy2 - biy) * (biz - biz1)
            + acicjck * (bix - bix1) * (biy - biy1) * (biz - biz1)
            + acifjck * (bix - bix1) * (biy2 - biy) * (biz - biz1)) * dxdydz;
}

}  // namespace afid
