/*
 * afid_cpu.c -- multi-threaded C restatement of AFiD's RK3 time step.
 *
 * TEST INFRASTRUCTURE ONLY: a second, compiled CPU restatement of the
 * reference's hot path, used as the timed CPU baseline of bench.py (all host
 * threads through OpenMP) and cross-checked against the NumPy oracle in the
 * CPU tests.  The product path never calls it.
 *
 * It follows the reference routine by routine, in the reference's order and
 * floating-point expression order (build it without FMA contraction):
 *   ExplicitTerms{VX,VY,VZ,Temp}.F90 -> ImplicitAndUpdate{VX,VY,VZ,Temp}.F90
 *   with SolveImpEqnUpdate_{X,YZ,Temp}.F90 (dgttrf/dgttrs order, the shared
 *   rhs array's wall row carried between solves) -> CalcLocalDivergence.F90
 *   -> SolvePressureCorrection.F90 (r2c y, c2c z, /(nym nzm), complex Thomas
 *   per mode with the (0,0) mode pinned, inverse transforms) ->
 *   CorrectVelocity.F90 -> CorrectPressure.F90, substeps per TimeMarcher.F90.
 * The FFTs are a plain mixed-radix (2, 3, 4, 5, 7) Stockham transform with
 * twiddles from libm in long double.
 *
 * Arrays are stored q[(k * nzm + i) * nym + j] (y fastest, then z, then x),
 * k over nx planes; periodic neighbours are index wraps.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int nxm, nym, nzm, nsst, inslws, inslwn;
  double alx3, ylen, zlen, ray, pra, tempbp, temptp;
} afid_cpu_params;

typedef struct {
  double re, im;
} cplx;

typedef struct {
  afid_cpu_params p;
  int nx, nxm, nym, nzm, nymh;
  long plane, fsize;
  double dx, dy, dz, dxq, dyq, dzq, ren, pec;
  double *xc, *g3rc, *g3rm, *udx3c, *udx3m;
  double *am3ck, *ac3ck, *ap3ck, *am3sk, *ac3sk, *ap3sk, *am3ssk, *ac3ssk, *ap3ssk;
  double *amphk, *acphk, *apphk, *ak1, *ak2;
  double *vx, *vy, *vz, *temp, *pr, *rux, *ruy, *ruz, *rutemp;
  double *rhs, *qcap, *dph, *dq, *hro;
  cplx *spec;
  cplx *twy, *twz;
  int rady[16], nry, radz[16], nrz;
} afid_cpu;

#define IDX(S, k, j, i) ((long)(k) * (S)->plane + (long)(i) * (S)->nym + (j))

static int factor(int n, int *rad) {
  int m = n, c = 0;
  while (m % 4 == 0) { rad[c++] = 4; m /= 4; }
  while (m % 2 == 0) { rad[c++] = 2; m /= 2; }
  for (int q = 3; q <= 7; q += 2)
    while (m % q == 0) { rad[c++] = q; m /= q; }
  return m == 1 ? c : -1;
}

static void twiddles(int n, cplx *w) {
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < n; ++k) {
    long double a = 2.0L * pi * (long double)k / (long double)n;
    w[k].re = (double)cosl(a);
    w[k].im = (double)(-sinl(a));
  }
}

/* In-place complex DFT of length n (sign -1 forward, +1 backward,
 * unnormalised), Stockham auto-sort with scratch b. */
static void fft(cplx *a, cplx *b, int n, const int *rad, int nr, const cplx *tw, int sgn) {
  int ns = 1;
  cplx *src = a, *dst = b;
  for (int p = 0; p < nr; ++p) {
    const int R = rad[p], nR = n / R, tstr = n / (ns * R);
    for (int j = 0; j < nR; ++j) {
      const int k = j % ns;
      cplx v[7], o[7];
      for (int r = 0; r < R; ++r) {
        cplx x = src[j + r * nR];
        if (r > 0 && k > 0) {
          cplx w = tw[r * k * tstr];
          if (sgn > 0) w.im = -w.im;
          cplx y = {x.re * w.re - x.im * w.im, x.re * w.im + x.im * w.re};
          x = y;
        }
        v[r] = x;
      }
      for (int q = 0; q < R; ++q) {
        cplx acc = v[0];
        for (int m = 1; m < R; ++m) {
          cplx w = tw[((m * q) % R) * (n / R)];
          if (sgn > 0) w.im = -w.im;
          acc.re += v[m].re * w.re - v[m].im * w.im;
          acc.im += v[m].re * w.im + v[m].im * w.re;
        }
        o[q] = acc;
      }
      const int base = (j / ns) * ns * R + k;
      for (int r = 0; r < R; ++r) dst[base + r * ns] = o[r];
    }
    cplx *t = src; src = dst; dst = t;
    ns *= R;
  }
  if (src != a) memcpy(a, src, sizeof(cplx) * (size_t)n);
}

static double *zalloc(long n) { return (double *)calloc((size_t)n, sizeof(double)); }

void afid_cpu_destroy(afid_cpu *S);

afid_cpu *afid_cpu_create(const afid_cpu_params *p, const double *xc_in) {
  if (p->nxm + 1 > 4096) return NULL;
  afid_cpu *S = (afid_cpu *)calloc(1, sizeof(afid_cpu));
  if (!S) return NULL;
  S->p = *p;
  const int nxm = p->nxm, nx = nxm + 1, nym = p->nym, nzm = p->nzm;
  S->nx = nx; S->nxm = nxm; S->nym = nym; S->nzm = nzm; S->nymh = nym / 2 + 1;
  S->plane = (long)nym * nzm;
  S->fsize = (long)nx * S->plane;
  S->nry = factor(nym, S->rady);
  S->nrz = factor(nzm, S->radz);
  if (S->nry < 0 || S->nrz < 0 || nym % 2) { free(S); return NULL; }
  const double pi = 2.0 * asin(1.0);
  S->dx = (double)nxm / p->alx3; S->dy = (double)nym / p->ylen; S->dz = (double)nzm / p->zlen;
  S->dxq = S->dx * S->dx; S->dyq = S->dy * S->dy; S->dzq = S->dz * S->dz;
  S->ren = sqrt(p->ray / p->pra); S->pec = sqrt(p->pra * p->ray);
  double **tabs[] = {&S->xc, &S->g3rc, &S->g3rm, &S->udx3c, &S->udx3m, &S->am3ck, &S->ac3ck, &S->ap3ck,
                     &S->am3sk, &S->ac3sk, &S->ap3sk, &S->am3ssk, &S->ac3ssk, &S->ap3ssk,
                     &S->amphk, &S->acphk, &S->apphk};
  for (unsigned q = 0; q < sizeof tabs / sizeof tabs[0]; ++q) *tabs[q] = zalloc(nx);
  S->ak1 = zalloc(nzm); S->ak2 = zalloc(nym);
  memcpy(S->xc, xc_in, sizeof(double) * nx);
  const double *xc = S->xc;
  const double dx = S->dx, dxq = S->dxq;
  /* CreateGrid.F90:143-266 */
  for (int kc = 1; kc <= nxm; ++kc) S->g3rm[kc - 1] = (xc[kc] - xc[kc - 1]) * dx;
  for (int kc = 2; kc <= nxm; ++kc) S->g3rc[kc - 1] = (xc[kc] - xc[kc - 2]) * dx * 0.5;
  S->g3rc[0] = (xc[1] - xc[0]) * dx;
  S->g3rc[nx - 1] = (xc[nx - 1] - xc[nxm - 1]) * dx;
  for (int kc = 1; kc <= nxm; ++kc) { S->udx3m[kc - 1] = dx / S->g3rm[kc - 1]; S->udx3c[kc - 1] = dx / S->g3rc[kc - 1]; }
  S->udx3c[nx - 1] = dx / S->g3rc[nx - 1];
  S->ac3ck[0] = 1.0; S->ac3ck[nx - 1] = 1.0;
  for (int kc = 2; kc <= nxm; ++kc) {
    double a33 = dxq / S->g3rc[kc - 1], a33p = 1.0 / S->g3rm[kc - 1], a33m = 1.0 / S->g3rm[kc - 2];
    S->ap3ck[kc - 1] = a33 * a33p; S->am3ck[kc - 1] = a33 * a33m;
    S->ac3ck[kc - 1] = -(S->ap3ck[kc - 1] + S->am3ck[kc - 1]);
  }
  for (int kc = 2; kc <= nxm - 1; ++kc) {
    double a33 = dxq / S->g3rm[kc - 1];
    S->ap3sk[kc - 1] = +a33 / S->g3rc[kc]; S->am3sk[kc - 1] = +a33 / S->g3rc[kc - 1];
    S->ac3sk[kc - 1] = -(S->ap3sk[kc - 1] + S->am3sk[kc - 1]);
  }
  {
    double a33 = dxq / S->g3rm[0], a33p = +a33 / S->g3rc[1], a33m = +a33 / S->g3rc[0];
    S->ap3sk[0] = a33p; S->am3sk[0] = 0.0; S->ac3sk[0] = -(a33p + p->inslws * a33m * 2.0);
    a33 = dxq / S->g3rm[nxm - 1]; a33p = +a33 / S->g3rc[nxm]; a33m = +a33 / S->g3rc[nxm - 1];
    S->am3sk[nxm - 1] = a33m; S->ap3sk[nxm - 1] = 0.0; S->ac3sk[nxm - 1] = -(a33m + p->inslwn * a33p * 2.0);
  }
  S->ac3ssk[0] = 1.0;
  for (int kc = 2; kc <= nxm; ++kc) {
    double a33 = dxq / S->g3rc[kc - 1], a33p = 1.0 / S->g3rm[kc - 1], a33m = 1.0 / S->g3rm[kc - 2];
    S->ap3ssk[kc - 1] = a33 * a33p; S->am3ssk[kc - 1] = a33 * a33m;
    S->ac3ssk[kc - 1] = -(S->ap3ssk[kc - 1] + S->am3ssk[kc - 1]);
  }
  S->ac3ssk[nx - 1] = 1.0;
  /* InitPressureSolver.F90:22-59 */
  for (int kc = 1; kc <= nxm; ++kc) {
    int kp = kc == nxm ? kc : kc + 1;
    double kmc = kc == 1 ? 0.0 : 1.0, kpc = kc == nxm ? 0.0 : 1.0;
    double a33icc = kmc * dxq / S->g3rc[kc - 1], a33icp = kpc * dxq / S->g3rc[kp - 1];
    double ugmmm = 1.0 / S->g3rm[kc - 1];
    S->amphk[kc - 1] = a33icc * ugmmm; S->apphk[kc - 1] = a33icp * ugmmm;
    S->acphk[kc - 1] = -(S->amphk[kc - 1] + S->apphk[kc - 1]);
  }
  for (int i = 1; i <= nzm; ++i) {
    double ao = i <= nzm / 2 + 1 ? (i - 1) * 2.0 * pi : -(nzm - i + 1) * 2.0 * pi;
    double f = (double)nzm / p->zlen;
    S->ak1[i - 1] = 2.0 * (1.0 - cos(ao / nzm)) * (f * f);
  }
  for (int j = 1; j <= nym; ++j) {
    double ap = j <= nym / 2 + 1 ? (j - 1) * 2.0 * pi : -(nym - j + 1) * 2.0 * pi;
    double f = (double)nym / p->ylen;
    S->ak2[j - 1] = 2.0 * (1.0 - cos(ap / nym)) * (f * f);
  }
  double **flds[] = {&S->vx, &S->vy, &S->vz, &S->temp, &S->pr, &S->rux, &S->ruy, &S->ruz, &S->rutemp,
                     &S->rhs, &S->qcap, &S->dph, &S->dq, &S->hro};
  for (unsigned q = 0; q < sizeof flds / sizeof flds[0]; ++q) {
    *flds[q] = zalloc(S->fsize);
    if (!*flds[q]) { afid_cpu_destroy(S); return NULL; }
  }
  S->spec = (cplx *)calloc((size_t)nxm * nzm * S->nymh, sizeof(cplx));
  S->twy = (cplx *)calloc(nym, sizeof(cplx));
  S->twz = (cplx *)calloc(nzm, sizeof(cplx));
  if (!S->spec || !S->twy || !S->twz) { afid_cpu_destroy(S); return NULL; }
  twiddles(nym, S->twy);
  twiddles(nzm, S->twz);
  return S;
}

void afid_cpu_destroy(afid_cpu *S) {
  if (!S) return;
  double *ps[] = {S->xc, S->g3rc, S->g3rm, S->udx3c, S->udx3m, S->am3ck, S->ac3ck, S->ap3ck, S->am3sk,
                  S->ac3sk, S->ap3sk, S->am3ssk, S->ac3ssk, S->ap3ssk, S->amphk, S->acphk, S->apphk,
                  S->ak1, S->ak2, S->vx, S->vy, S->vz, S->temp, S->pr, S->rux, S->ruy, S->ruz, S->rutemp,
                  S->rhs, S->qcap, S->dph, S->dq, S->hro};
  for (unsigned q = 0; q < sizeof ps / sizeof ps[0]; ++q) free(ps[q]);
  free(S->spec); free(S->twy); free(S->twz);
  free(S);
}

/* field ids as the C-ABI of the library: 0 vx 1 vy 2 vz 3 temp 4 pr 9 dph 14 wall(rhs row 1) */
static double *field(afid_cpu *S, int f) {
  switch (f) {
    case 0: return S->vx; case 1: return S->vy; case 2: return S->vz; case 3: return S->temp;
    case 4: return S->pr; case 5: return S->rux; case 6: return S->ruy; case 7: return S->ruz;
    case 8: return S->rutemp; case 9: return S->dph; default: return NULL;
  }
}

/* Copy a field in or out; host arrays in the layout q[k][i][j] (y fastest). */
int afid_cpu_set(afid_cpu *S, int f, const double *a) {
  double *d = field(S, f);
  if (!d) return -1;
  memcpy(d, a, sizeof(double) * (size_t)(f == 9 ? S->nxm * S->plane : S->fsize));
  return 0;
}
int afid_cpu_get(afid_cpu *S, int f, double *a) {
  double *d = field(S, f);
  if (!d) return -1;
  memcpy(a, d, sizeof(double) * (size_t)(f == 9 ? S->nxm * S->plane : S->fsize));
  return 0;
}

#define W(a, n) (((a) + (n)) % (n))

/* ---- explicit terms (ExplicitTerms*.F90) ---------------------------------- */
static void explicit_terms(afid_cpu *S) {
  const int nxm = S->nxm, nym = S->nym, nzm = S->nzm;
  const double udy = S->dy * 0.25, udz = S->dz * 0.25;
  const double udyq = S->dyq / S->ren, udzq = S->dzq / S->ren;
  const double tudyq = S->dyq / S->pec, tudzq = S->dzq / S->pec;
  const double *vx = S->vx, *vy = S->vy, *vz = S->vz, *t = S->temp;
#pragma omp parallel for collapse(2) schedule(static)
  for (int kc = 0; kc < nxm; ++kc)
    for (int i = 0; i < nzm; ++i) {
      const int im = W(i - 1, nzm), ip = W(i + 1, nzm);
      for (int j = 0; j < nym; ++j) {
        const int jm = W(j - 1, nym), jp = W(j + 1, nym);
        const int km = kc - 1, kp = kc + 1;
        const int kmm = kc == 0 ? 0 : kc - 1, kpp = kc == nxm - 1 ? kc : kc + 1;
#define A(q, k, jj, ii) q[IDX(S, k, jj, ii)]
        if (kc >= 1) {
          /* ExplicitTermsVX.F90:55-101 */
          double hxz = (((A(vz, kc, j, ip) + A(vz, km, j, ip)) * (A(vx, kc, j, ip) + A(vx, kc, j, i)))
                        - ((A(vz, kc, j, i) + A(vz, km, j, i)) * (A(vx, kc, j, i) + A(vx, kc, j, im)))) * udz;
          double hxy = (((A(vy, kc, jp, i) + A(vy, km, jp, i)) * (A(vx, kc, jp, i) + A(vx, kc, j, i)))
                        - ((A(vy, kc, j, i) + A(vy, km, j, i)) * (A(vx, kc, j, i) + A(vx, kc, jm, i)))) * udy;
          double pp = A(vx, kp, j, i) + A(vx, kc, j, i), mm = A(vx, kc, j, i) + A(vx, km, j, i);
          double hxx = (pp * pp - mm * mm) * S->udx3c[kc] * 0.25;
          double dzzvx = (A(vx, kc, j, im) - 2.0 * A(vx, kc, j, i) + A(vx, kc, j, ip)) * udzq;
          double dyyvx = (A(vx, kc, jm, i) - 2.0 * A(vx, kc, j, i) + A(vx, kc, jp, i)) * udyq;
          S->qcap[IDX(S, kc, j, i)] = -(hxx + hxy + hxz) + dyyvx + dzzvx + A(t, kc, j, i);
          /* ExplicitTermsTemp.F90:52-93 */
          double htz = ((A(vz, km, j, ip) + A(vz, kc, j, ip)) * (A(t, kc, j, ip) + A(t, kc, j, i))
                        - (A(vz, km, j, i) + A(vz, kc, j, i)) * (A(t, kc, j, i) + A(t, kc, j, im))) * udz;
          double hty = ((A(vy, kc, jp, i) + A(vy, km, jp, i)) * (A(t, kc, jp, i) + A(t, kc, j, i))
                        - (A(vy, kc, j, i) + A(vy, km, j, i)) * (A(t, kc, j, i) + A(t, kc, jm, i))) * udy;
          double htx = ((A(vx, kp, j, i) + A(vx, kc, j, i)) * (A(t, kp, j, i) + A(t, kc, j, i))
                        - (A(vx, kc, j, i) + A(vx, km, j, i)) * (A(t, kc, j, i) + A(t, km, j, i))) * S->udx3c[kc] * 0.25;
          double dzzt = (A(t, kc, j, ip) - 2.0 * A(t, kc, j, i) + A(t, kc, j, im)) * tudzq;
          double dyyt = (A(t, kc, jp, i) - 2.0 * A(t, kc, j, i) + A(t, kc, jm, i)) * tudyq;
          S->hro[IDX(S, kc, j, i)] = -(htx + hty + htz) + dyyt + dzzt;
        }
        /* ExplicitTermsVY.F90:54-98 */
        {
          double vyc = A(vy, kc, j, i);
          double hyx = ((A(vx, kp, j, i) + A(vx, kp, jm, i)) * (A(vy, kpp, j, i) + vyc)
                        - (A(vx, kc, j, i) + A(vx, kc, jm, i)) * (vyc + A(vy, kmm, j, i))) * S->udx3m[kc] * 0.25;
          double pp = A(vy, kc, jp, i) + vyc, mm = A(vy, kc, jm, i) + vyc;
          double hyy = (pp * pp - mm * mm) * udy;
          double hyz = ((A(vy, kc, j, ip) + vyc) * (A(vz, kc, j, ip) + A(vz, kc, jm, ip))
                        - (vyc + A(vy, kc, j, im)) * (A(vz, kc, j, i) + A(vz, kc, jm, i))) * udz;
          double dyyvy = (A(vy, kc, jp, i) - 2.0 * vyc + A(vy, kc, jm, i)) * udyq;
          double dzzvy = (A(vy, kc, j, ip) - 2.0 * vyc + A(vy, kc, j, im)) * udzq;
          S->dph[IDX(S, kc, j, i)] = -(hyx + hyy + hyz) + dyyvy + dzzvy;
        }
        /* ExplicitTermsVZ.F90:56-101 */
        {
          double vzc = A(vz, kc, j, i);
          double pp = A(vz, kc, j, ip) + vzc, mm = A(vz, kc, j, im) + vzc;
          double hzz = (pp * pp - mm * mm) * udz;
          double hzy = ((A(vy, kc, jp, i) + A(vy, kc, jp, im)) * (A(vz, kc, jp, i) + vzc)
                        - (A(vy, kc, j, i) + A(vy, kc, j, im)) * (vzc + A(vz, kc, jm, i))) * udy;
          double hzx = ((A(vx, kp, j, i) + A(vx, kp, j, im)) * (A(vz, kpp, j, i) + vzc)
                        - (A(vx, kc, j, i) + A(vx, kc, j, im)) * (vzc + A(vz, kmm, j, i))) * S->udx3m[kc] * 0.25;
          double dzzvz = (A(vz, kc, j, ip) - 2.0 * vzc + A(vz, kc, j, im)) * udzq;
          double dyyvz = (A(vz, kc, jp, i) - 2.0 * vzc + A(vz, kc, jm, i)) * udyq;
          S->dq[IDX(S, kc, j, i)] = -(hzx + hzy + hzz) + dyyvz + dzzvz;
        }
#undef A
      }
    }
}

/* ---- tridiagonal (dgttrf/dgttrs without pivoting, diagonally dominant) ---- */
typedef struct {
  double sc[4096], fact[4096], dp[4096], du[4096];
  int n, k0;   /* system size, first updated row */
} tri;

/* size-n system with rows am/ap from the metric arrays scaled as in
 * SolveImpEqnUpdate_*: row k = [-am*bx*s, 1, -ap*bx*s], s = 1/(1 - ac*bx);
 * rows outside [lo, hi] are identity rows */
static void tri_factor(tri *T, int n, int lo, int hi, const double *am, const double *ac,
                       const double *ap, double bx) {
  double dl[4097], d[4097];
  T->n = n;
  for (int k = 0; k < n; ++k) {
    double s = 1.0, a = 0.0, c = 0.0;
    if (k >= lo && k <= hi) {
      s = 1.0 / (1.0 - ac[k] * bx);
      a = -am[k] * bx * s;
      c = -ap[k] * bx * s;
    }
    T->sc[k] = s; dl[k] = a; T->du[k] = c; d[k] = 1.0;
  }
  T->dp[0] = 1.0;
  T->fact[0] = 0.0;
  for (int k = 0; k < n - 1; ++k) {
    double fact = dl[k + 1] / d[k];
    d[k + 1] = d[k + 1] - fact * T->du[k];
    T->fact[k + 1] = fact;
    T->dp[k + 1] = d[k + 1];
  }
}

static void implicit_update(afid_cpu *S, double al, double ga, double ro, double dt, double beta) {
  const int nx = S->nx, nxm = S->nxm, nym = S->nym, nzm = S->nzm;
  const long P = S->plane;
  static tri TX, TY, TT;
  const double bx = beta * al;
  tri_factor(&TX, nx, 1, nxm - 1, S->am3ssk, S->ac3ck, S->ap3ssk, bx);
  tri_factor(&TY, nxm, 0, nxm - 1, S->am3sk, S->ac3sk, S->ap3sk, bx);
  tri_factor(&TT, nx, 1, nxm - 1, S->am3ssk, S->ac3ssk, S->ap3ssk, 0.5 * al * dt / S->pec);
  const double alre = al / S->ren, alpec = al / S->pec, udyal = S->dy * al;
  double *rhs = S->rhs;
  /* per z-row i: every sweep runs over k with the contiguous y index
   * innermost; each column still sees VX, VY, VZ, Temp in the reference's
   * order, so the shared rhs array behaves as in the reference */
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nzm; ++i) {
    const long r0 = (long)i * nym;
    const int im = W(i - 1, nzm);
#define ROW(k) ((long)(k) * P + r0)
    /* ImplicitAndUpdateVX.F90:37-77 with SolveImpEqnUpdate_X.F90 */
    for (int k = 1; k < nxm; ++k)
      for (int j = 0; j < nym; ++j) {
        const long o = ROW(k) + j;
        double dxx = S->vx[o + P] * S->ap3ck[k] + S->vx[o] * S->ac3ck[k] + S->vx[o - P] * S->am3ck[k];
        double dxp = (S->pr[o] - S->pr[o - P]) * (al * S->udx3c[k]);
        rhs[o] = (ga * S->qcap[o] + ro * S->rux[o] + alre * dxx - dxp) * dt;
        S->rux[o] = S->qcap[o];
        rhs[o] = rhs[o] * TX.sc[k];
      }
    for (int k = 1; k < nx; ++k)
      for (int j = 0; j < nym; ++j) rhs[ROW(k) + j] = rhs[ROW(k) + j] - TX.fact[k] * rhs[ROW(k - 1) + j];
    for (int j = 0; j < nym; ++j) rhs[ROW(nx - 1) + j] = rhs[ROW(nx - 1) + j] / TX.dp[nx - 1];
    for (int k = nx - 2; k >= 0; --k)
      for (int j = 0; j < nym; ++j)
        rhs[ROW(k) + j] = (rhs[ROW(k) + j] - TX.du[k] * rhs[ROW(k + 1) + j]) / TX.dp[k];
    for (int k = 1; k < nxm; ++k)
      for (int j = 0; j < nym; ++j) S->vx[ROW(k) + j] += rhs[ROW(k) + j];
    for (int j = 0; j < nym; ++j) { S->vx[ROW(0) + j] = 0.0; S->vx[ROW(nx - 1) + j] = 0.0; }
    /* ImplicitAndUpdateVY/VZ.F90 with SolveImpEqnUpdate_YZ.F90 */
    for (int f = 0; f < 2; ++f) {
      double *q = f == 0 ? S->vy : S->vz;
      double *hnew = f == 0 ? S->dph : S->dq;
      double *hold = f == 0 ? S->ruy : S->ruz;
      for (int k = 0; k < nxm; ++k) {
        const int kmm = k == 0 ? 0 : k - 1, kpp = k == nxm - 1 ? k : k + 1;
        for (int j = 0; j < nym; ++j) {
          const long o = ROW(k) + j;
          const int jm = W(j - 1, nym);
          double dxx = q[ROW(kpp) + j] * S->ap3sk[k] + q[o] * S->ac3sk[k] + q[ROW(kmm) + j] * S->am3sk[k];
          double dp = f == 0 ? (S->pr[o] - S->pr[ROW(k) + jm]) * udyal
                             : (S->pr[o] - S->pr[(long)k * P + (long)im * nym + j]) * S->dz * al;
          rhs[o] = (ga * hnew[o] + ro * hold[o] + alre * dxx - dp) * dt;
          hold[o] = hnew[o];
          rhs[o] = rhs[o] * TY.sc[k];
        }
      }
      for (int k = 1; k < nxm; ++k)
        for (int j = 0; j < nym; ++j) rhs[ROW(k) + j] = rhs[ROW(k) + j] - TY.fact[k] * rhs[ROW(k - 1) + j];
      for (int j = 0; j < nym; ++j) rhs[ROW(nxm - 1) + j] = rhs[ROW(nxm - 1) + j] / TY.dp[nxm - 1];
      for (int k = nxm - 2; k >= 0; --k)
        for (int j = 0; j < nym; ++j)
          rhs[ROW(k) + j] = (rhs[ROW(k) + j] - TY.du[k] * rhs[ROW(k + 1) + j]) / TY.dp[k];
      for (int k = 0; k < nxm; ++k)
        for (int j = 0; j < nym; ++j) q[ROW(k) + j] += rhs[ROW(k) + j];
    }
    /* ImplicitAndUpdateTemp.F90 with SolveImpEqnUpdate_Temp.F90 */
    for (int k = 1; k < nxm; ++k)
      for (int j = 0; j < nym; ++j) {
        const long o = ROW(k) + j;
        double dxx = S->temp[o + P] * S->ap3ck[k] + S->temp[o] * S->ac3ck[k] + S->temp[o - P] * S->am3ck[k];
        rhs[o] = (ga * S->hro[o] + ro * S->rutemp[o] + alpec * dxx) * dt;
        S->rutemp[o] = S->hro[o];
        rhs[o] = rhs[o] * TT.sc[k];
      }
    for (int k = 1; k < nx; ++k)
      for (int j = 0; j < nym; ++j) rhs[ROW(k) + j] = rhs[ROW(k) + j] - TT.fact[k] * rhs[ROW(k - 1) + j];
    for (int j = 0; j < nym; ++j) rhs[ROW(nx - 1) + j] = rhs[ROW(nx - 1) + j] / TT.dp[nx - 1];
    for (int k = nx - 2; k >= 0; --k)
      for (int j = 0; j < nym; ++j)
        rhs[ROW(k) + j] = (rhs[ROW(k) + j] - TT.du[k] * rhs[ROW(k + 1) + j]) / TT.dp[k];
    for (int k = 1; k < nxm; ++k)
      for (int j = 0; j < nym; ++j) S->temp[ROW(k) + j] += rhs[ROW(k) + j];
    for (int j = 0; j < nym; ++j) { S->temp[ROW(0) + j] = S->p.tempbp; S->temp[ROW(nx - 1) + j] = S->p.temptp; }
#undef ROW
  }
}

/* ---- pressure (CalcLocalDivergence, SolvePressureCorrection) -------------- */
static void pressure(afid_cpu *S, double al, double dt) {
  const int nxm = S->nxm, nym = S->nym, nzm = S->nzm, nh = S->nymh;
  const long P = S->plane;
  const double usdtal = 1.0 / (dt * al);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nxm; ++k)
    for (int i = 0; i < nzm; ++i)
      for (int j = 0; j < nym; ++j) {
        const long o = IDX(S, k, j, i);
        double dq = (S->vz[IDX(S, k, j, W(i + 1, nzm))] - S->vz[o]) * S->dz
                  + (S->vy[IDX(S, k, W(j + 1, nym), i)] - S->vy[o]) * S->dy
                  + (S->vx[o + P] - S->vx[o]) * S->udx3m[k];
        S->dph[o] = dq * usdtal;
      }
  /* r2c along y */
#pragma omp parallel
  {
    cplx *a = (cplx *)malloc(sizeof(cplx) * (nym > nzm ? nym : nzm));
    cplx *b = (cplx *)malloc(sizeof(cplx) * (nym > nzm ? nym : nzm));
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nxm; ++k)
      for (int i = 0; i < nzm; ++i) {
        for (int j = 0; j < nym; ++j) { a[j].re = S->dph[IDX(S, k, j, i)]; a[j].im = 0.0; }
        fft(a, b, nym, S->rady, S->nry, S->twy, -1);
        for (int q = 0; q < nh; ++q) S->spec[((long)k * nzm + i) * nh + q] = a[q];
      }
    /* c2c along z, normalise */
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nxm; ++k)
      for (int q = 0; q < nh; ++q) {
        for (int i = 0; i < nzm; ++i) a[i] = S->spec[((long)k * nzm + i) * nh + q];
        fft(a, b, nzm, S->radz, S->nrz, S->twz, -1);
        const double nrm = (double)(nzm * nym);
        for (int i = 0; i < nzm; ++i) {
          cplx v = a[i];
          v.re = v.re / nrm; v.im = v.im / nrm;
          S->spec[((long)k * nzm + i) * nh + q] = v;
        }
      }
    free(a); free(b);
  }
  /* complex tridiagonal per mode (SolvePressureCorrection.F90:117-137) */
  const long nmode = (long)nzm * nh;
#pragma omp parallel
  {
    double *d = (double *)malloc(sizeof(double) * nxm);
#pragma omp for schedule(static)
    for (long m = 0; m < nmode; ++m) {
      const int kz = (int)(m / nh), ky = (int)(m % nh);
      const double ak = S->ak2[ky], a1 = S->ak1[kz];
      cplx *x = S->spec + m;
      double s = 1.0 / ((S->acphk[0] - ak) - a1);
      cplx y = x[0];
      y.re *= s; y.im *= s;
      double dd = 1.0, apv = S->apphk[0] * s;
      x[0] = y; d[0] = 1.0;
      for (int k = 1; k < nxm; ++k) {
        s = 1.0 / ((S->acphk[k] - ak) - a1);
        double am = S->amphk[k] * s, fact = am / dd;
        dd = 1.0 - fact * apv;
        cplx r = x[(long)k * nmode];
        r.re *= s; r.im *= s;
        y.re = r.re - fact * y.re; y.im = r.im - fact * y.im;
        x[(long)k * nmode] = y; d[k] = dd;
        apv = S->apphk[k] * s;
      }
      cplx xn = {0.0, 0.0};
      if (!(ky == 0 && kz == 0)) { xn.re = y.re / dd; xn.im = y.im / dd; }
      x[(long)(nxm - 1) * nmode] = xn;
      for (int k = nxm - 2; k >= 0; --k) {
        double sk = 1.0 / ((S->acphk[k] - ak) - a1), ap = S->apphk[k] * sk;
        cplx yk = x[(long)k * nmode];
        xn.re = (yk.re - ap * xn.re) / d[k];
        xn.im = (yk.im - ap * xn.im) / d[k];
        x[(long)k * nmode] = xn;
      }
    }
    free(d);
  }
  /* inverse z, then c2r along y */
#pragma omp parallel
  {
    cplx *a = (cplx *)malloc(sizeof(cplx) * (nym > nzm ? nym : nzm));
    cplx *b = (cplx *)malloc(sizeof(cplx) * (nym > nzm ? nym : nzm));
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nxm; ++k)
      for (int q = 0; q < nh; ++q) {
        for (int i = 0; i < nzm; ++i) a[i] = S->spec[((long)k * nzm + i) * nh + q];
        fft(a, b, nzm, S->radz, S->nrz, S->twz, +1);
        for (int i = 0; i < nzm; ++i) S->spec[((long)k * nzm + i) * nh + q] = a[i];
      }
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nxm; ++k)
      for (int i = 0; i < nzm; ++i) {
        const cplx *c = S->spec + ((long)k * nzm + i) * nh;
        for (int n = 0; n < nym; ++n) {
          int q = n < nh ? n : nym - n;
          cplx v = c[q];
          if (q == 0 || 2 * q == nym) v.im = 0.0;
          else if (n >= nh) v.im = -v.im;
          a[n] = v;
        }
        fft(a, b, nym, S->rady, S->nry, S->twy, +1);
        for (int j = 0; j < nym; ++j) S->dph[IDX(S, k, j, i)] = a[j].re;
      }
    free(a); free(b);
  }
}

/* ---- projection (CorrectVelocity, CorrectPressure) ------------------------ */
static void correct(afid_cpu *S, double al, double dt, double beta) {
  const int nxm = S->nxm, nym = S->nym, nzm = S->nzm;
  const long P = S->plane;
  const double udy = al * dt * S->dy, udz = al * dt * S->dz, be = al * beta;
  const double *f = S->dph;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nxm; ++k)
    for (int i = 0; i < nzm; ++i) {
      const int im = W(i - 1, nzm), ip = W(i + 1, nzm);
      const int km = k == 0 ? 0 : k - 1, kp = k == nxm - 1 ? k : k + 1;
      const double usukm = al * dt * S->udx3c[k];
      for (int j = 0; j < nym; ++j) {
        const int jm = W(j - 1, nym), jp = W(j + 1, nym);
        const long o = IDX(S, k, j, i);
        const double fc = f[o];
        if (k >= 1) S->vx[o] = S->vx[o] - (fc - f[IDX(S, km, j, i)]) * usukm;
        S->vy[o] = S->vy[o] - (fc - f[IDX(S, k, jm, i)]) * udy;
        S->vz[o] = S->vz[o] - (fc - f[IDX(S, k, j, im)]) * udz;
        S->pr[o] = S->pr[o] + fc - be * ((f[IDX(S, k, j, ip)] - 2.0 * fc + f[IDX(S, k, j, im)]) * S->dzq
                                        + (f[IDX(S, k, jp, i)] - 2.0 * fc + f[IDX(S, k, jm, i)]) * S->dyq
                                        + (f[IDX(S, kp, j, i)] * S->apphk[k] + fc * S->acphk[k]
                                           + f[IDX(S, km, j, i)] * S->amphk[k]));
      }
    }
}

/* One TimeMarcher step (TimeMarcher.F90:22-74) with a fixed dt. */
void afid_cpu_step(afid_cpu *S, double dt, int nsteps) {
  double gam[3], rom[3];
  if (S->p.nsst > 1) { gam[0] = 8.0 / 15.0; gam[1] = 5.0 / 12.0; gam[2] = 3.0 / 4.0;
                       rom[0] = 0.0; rom[1] = -17.0 / 60.0; rom[2] = -5.0 / 12.0; }
  else { gam[0] = 1.5; gam[1] = 0.0; gam[2] = 0.0; rom[0] = -0.5; rom[1] = 0.0; rom[2] = 0.0; }
  for (int st = 0; st < nsteps; ++st) {
    const double beta = dt / S->ren * 0.5;
    for (int ns = 0; ns < S->p.nsst; ++ns) {
      const double al = gam[ns] + rom[ns];
      explicit_terms(S);
      implicit_update(S, al, gam[ns], rom[ns], dt, beta);
      pressure(S, al, dt);
      correct(S, al, dt, beta);
    }
  }
}
