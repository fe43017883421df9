/*
 * afid_cpu.c — CPU restatement (C + OpenMP) of AFiD's RK3 flow + temperature substep.
 * TEST INFRASTRUCTURE ONLY: the timed CPU baseline of bench.py and a second oracle beside the
 * NumPy oracle (oracle/afid_oracle.py), which it is tested against.  Never part of the
 * product path.
 *
 * It follows the same reference routines as the NumPy oracle, one loop nest per routine:
 *   ExplicitTerms{VX,VY,VZ,Temp}.F90, ImplicitAndUpdate{VX,VY,VZ,Temp}.F90,
 *   SolveImpEqnUpdate_{X,YZ,Temp}.F90 (LAPACK dgttrf/dgttrs restated below),
 *   pressure.F90:141-301 (y r2c / z c2c FFT restated as a mixed-radix FFT, zgttrf/zgttrs per
 *   mode with the 1+1e-15 diagonal), CalcMaxCFL.F90:30-43, TimeMarcher.F90:28-133.
 * Layout: x fastest, (k, j, i) at k + nx*(j + nym*i), periodic y/z by index wrap.
 * The reference's 2DECOMP pencils are replaced by OpenMP loops over independent lines.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;

typedef struct {
  int nxm, nym, nzm, nx, nsst;
  double dy, dz, dyq, dzq, ren, pect, byct, gy, xplusu, xminusu;
  int active_t, gaxis, inslws, inslwn, tfixs, tfixn;
  /* tables (0-based copies of the reference arrays) */
  double *udx3c, *udx3m, *idx, *ap3ck, *ac3ck, *am3ck, *ap3sk, *ac3sk, *am3sk, *ap3ssk, *ac3ssk,
      *am3ssk, *amphk, *acphk, *apphk, *ak1, *ak2, *tempbp, *temptp, *g3rc;
  /* state */
  double *vx, *vy, *vz, *temp, *pr, *rux, *ruy, *ruz, *rut;
  double *qcap, *dph, *dq, *hro, *phi;
  cplx *spec; /* (k, ky, i) with k fastest, ky < nym/2+1 */
  cplx *twy, *twz;
  int fy[32], nfy, fz[32], nfz;
} afid_cpu_t;

static size_t IDX(const afid_cpu_t *c, int k, int j, int i) {
  return (size_t)k + (size_t)c->nx * ((size_t)j + (size_t)c->nym * i);
}
static int wp(int a, int n) { return a + 1 == n ? 0 : a + 1; }
static int wm(int a, int n) { return a == 0 ? n - 1 : a - 1; }

static double *dup(const double *s, int n) {
  double *d = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  memcpy(d, s, sizeof(double) * n);
  return d;
}

static int factor(int n, int *f) {
  int m = n, c = 0;
  while (m % 4 == 0) { f[c++] = 4; m /= 4; }
  while (m % 2 == 0) { f[c++] = 2; m /= 2; }
  while (m % 3 == 0) { f[c++] = 3; m /= 3; }
  while (m % 5 == 0) { f[c++] = 5; m /= 5; }
  return m == 1 ? c : -1;
}

static cplx *make_tw(int n) {
  cplx *t = (cplx *)malloc(sizeof(cplx) * (n > 0 ? n : 1));
  for (int m = 0; m < n; ++m) {
    double a = 2.0 * M_PI * (double)m / (double)n;
    t[m] = cos(a) - I * sin(a);
  }
  return t;
}

/* exp(-+2 pi i e/R) for R <= 5, filled once */
static cplx g_root[2][6][5];
static void init_roots(void) {
  for (int inv = 0; inv < 2; ++inv)
    for (int R = 1; R <= 5; ++R)
      for (int e = 0; e < R; ++e) {
        double ang = 2.0 * M_PI * e / R;
        g_root[inv][R][e] = cos(ang) + (inv ? 1.0 : -1.0) * I * sin(ang);
      }
}

/* Stockham mixed-radix FFT of one sequence (sign -1 forward, +1 backward, unnormalised). */
static void fft1(cplx *x, cplx *w, int n, const int *f, int nf, const cplx *tw, int inv) {
  cplx *in = x, *out = w;
  int ns = 1;
  for (int p = 0; p < nf; ++p) {
    int R = f[p], nr = n / R, ts = n / (ns * R);
    for (int jj = 0; jj < nr; ++jj) {
      int k = jj % ns;
      cplx a[5];
      for (int q = 0; q < R; ++q) {
        a[q] = in[jj + q * nr];
        if (q && ns > 1) {
          cplx t = tw[q * k * ts];
          a[q] *= inv ? conj(t) : t;
        }
      }
      cplx *d = out + (jj / ns) * ns * R + k;
      const cplx *rt = g_root[inv ? 1 : 0][R];
      for (int q = 0; q < R; ++q) {
        cplx s = 0;
        for (int r = 0; r < R; ++r) s += a[r] * rt[(q * r) % R];
        d[q * ns] = s;
      }
    }
    cplx *t = in; in = out; out = t;
    ns *= R;
  }
  if (in != x) memcpy(x, in, sizeof(cplx) * n);
}

/* LAPACK dgttrf restated: LU of a tridiagonal with partial pivoting (dl, d, du, du2, ipiv). */
static int gttrf(int n, double *dl, double *d, double *du, double *du2, int *ipiv) {
  for (int i = 0; i < n; ++i) ipiv[i] = i;
  for (int i = 0; i < n - 2; ++i) du2[i] = 0.0;
  for (int i = 0; i < n - 2; ++i) {
    if (fabs(d[i]) >= fabs(dl[i])) {
      if (d[i] != 0.0) {
        double fact = dl[i] / d[i];
        dl[i] = fact;
        d[i + 1] = d[i + 1] - fact * du[i];
      }
    } else {
      double fact = d[i] / dl[i];
      d[i] = dl[i];
      dl[i] = fact;
      double temp = du[i];
      du[i] = d[i + 1];
      d[i + 1] = temp - fact * d[i + 1];
      du2[i] = du[i + 1];
      du[i + 1] = -fact * du[i + 1];
      ipiv[i] = i + 1;
    }
  }
  if (n > 1) {
    int i = n - 2;
    if (fabs(d[i]) >= fabs(dl[i])) {
      if (d[i] != 0.0) {
        double fact = dl[i] / d[i];
        dl[i] = fact;
        d[i + 1] = d[i + 1] - fact * du[i];
      }
    } else {
      double fact = d[i] / dl[i];
      d[i] = dl[i];
      dl[i] = fact;
      double temp = du[i];
      du[i] = d[i + 1];
      d[i + 1] = temp - fact * d[i + 1];
      ipiv[i] = i + 1;
    }
  }
  for (int i = 0; i < n; ++i)
    if (d[i] == 0.0) return i + 1;
  return 0;
}

/* LAPACK dgttrs ('N') restated for one right-hand side, real or complex. */
#define GTTRS_BODY(T)                                                              \
  for (int i = 0; i < n - 1; ++i) {                                                \
    if (ipiv[i] == i) {                                                            \
      b[i + 1] = b[i + 1] - dl[i] * b[i];                                          \
    } else {                                                                       \
      T temp = b[i];                                                               \
      b[i] = b[i + 1];                                                             \
      b[i + 1] = temp - dl[i] * b[i];                                              \
    }                                                                              \
  }                                                                                \
  b[n - 1] = b[n - 1] / d[n - 1];                                                  \
  if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];              \
  for (int i = n - 3; i >= 0; --i)                                                 \
    b[i] = (b[i] - du[i] * b[i + 1] - du2[i] * b[i + 2]) / d[i];

static void gttrs_r(int n, const double *dl, const double *d, const double *du, const double *du2,
                    const int *ipiv, double *b) {
  GTTRS_BODY(double)
}
static void gttrs_c(int n, const double *dl, const double *d, const double *du, const double *du2,
                    const int *ipiv, cplx *b) {
  GTTRS_BODY(cplx)
}

afid_cpu_t *afid_cpu_create(int nxm, int nym, int nzm, double ylen, double zlen, const double *tab[19],
                            const double *params, const int *iparams) {
  init_roots();
  afid_cpu_t *c = (afid_cpu_t *)calloc(1, sizeof(afid_cpu_t));
  c->nxm = nxm; c->nym = nym; c->nzm = nzm; c->nx = nxm + 1;
  int nx = nxm + 1;
  c->dy = (double)nym / ylen; c->dz = (double)nzm / zlen;
  c->dyq = c->dy * c->dy; c->dzq = c->dz * c->dz;
  c->ren = params[0]; c->pect = params[1]; c->byct = params[2];
  c->xplusu = params[3]; c->xminusu = params[4];
  double dpdy = params[5];
  c->active_t = iparams[0]; c->gaxis = iparams[1]; c->inslws = iparams[2]; c->inslwn = iparams[3];
  c->tfixs = iparams[4]; c->tfixn = iparams[5]; c->nsst = iparams[6];
  c->gy = (c->inslwn == 0 || c->inslws == 0) ? dpdy * dpdy / (c->ren * c->ren)
                                             : 8.0 * (dpdy * dpdy) / (c->ren * c->ren);
  /* tab order: udx3c udx3m ap3ck ac3ck am3ck ap3sk ac3sk am3sk ap3ssk ac3ssk am3ssk amphk acphk
     apphk ak1 ak2 tempbp temptp g3rc */
  c->udx3c = dup(tab[0], nx); c->udx3m = dup(tab[1], nx);
  c->ap3ck = dup(tab[2], nx); c->ac3ck = dup(tab[3], nx); c->am3ck = dup(tab[4], nx);
  c->ap3sk = dup(tab[5], nx); c->ac3sk = dup(tab[6], nx); c->am3sk = dup(tab[7], nx);
  c->ap3ssk = dup(tab[8], nx); c->ac3ssk = dup(tab[9], nx); c->am3ssk = dup(tab[10], nx);
  c->amphk = dup(tab[11], nx); c->acphk = dup(tab[12], nx); c->apphk = dup(tab[13], nx);
  c->ak1 = dup(tab[14], nzm); c->ak2 = dup(tab[15], nym);
  c->tempbp = dup(tab[16], nym * nzm); c->temptp = dup(tab[17], nym * nzm);
  c->g3rc = dup(tab[18], nx);
  c->idx = (double *)malloc(sizeof(double) * nx);
  for (int k = 0; k < nxm; ++k) c->idx[k] = 1.0 / c->udx3m[k];
  size_t n = (size_t)nx * nym * nzm;
  double **f[] = {&c->vx, &c->vy, &c->vz, &c->temp, &c->pr, &c->rux, &c->ruy, &c->ruz, &c->rut,
                  &c->qcap, &c->dph, &c->dq, &c->hro, &c->phi};
  for (size_t q = 0; q < sizeof f / sizeof f[0]; ++q) *f[q] = (double *)calloc(n, sizeof(double));
  c->spec = (cplx *)calloc((size_t)nxm * (nym / 2 + 1) * nzm, sizeof(cplx));
  c->nfy = factor(nym, c->fy);
  c->nfz = factor(nzm, c->fz);
  c->twy = make_tw(nym);
  c->twz = make_tw(nzm);
  if (c->nfy < 0 || c->nfz < 0) { free(c); return NULL; }
  return c;
}

void afid_cpu_destroy(afid_cpu_t *c) {
  if (!c) return;
  double *a[] = {c->udx3c, c->udx3m, c->idx, c->ap3ck, c->ac3ck, c->am3ck, c->ap3sk, c->ac3sk, c->am3sk,
                 c->ap3ssk, c->ac3ssk, c->am3ssk, c->amphk, c->acphk, c->apphk, c->ak1, c->ak2,
                 c->tempbp, c->temptp, c->g3rc, c->vx, c->vy, c->vz, c->temp, c->pr, c->rux, c->ruy, c->ruz,
                 c->rut, c->qcap, c->dph, c->dq, c->hro, c->phi};
  for (size_t q = 0; q < sizeof a / sizeof a[0]; ++q) free(a[q]);
  free(c->spec); free(c->twy); free(c->twz);
  free(c);
}

int afid_cpu_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* state arrays in the same (i, j, k) layout, nx per column; which: 0 vx 1 vy 2 vz 3 temp 4 pr */
void afid_cpu_set(afid_cpu_t *c, int which, const double *src) {
  double *d[] = {c->vx, c->vy, c->vz, c->temp, c->pr};
  memcpy(d[which], src, sizeof(double) * (size_t)c->nx * c->nym * c->nzm);
  if (which == 0) {
    size_t n = (size_t)c->nx * c->nym * c->nzm;
    memset(c->rux, 0, n * 8); memset(c->ruy, 0, n * 8); memset(c->ruz, 0, n * 8); memset(c->rut, 0, n * 8);
  }
}
void afid_cpu_get(const afid_cpu_t *c, int which, double *dst) {
  const double *d[] = {c->vx, c->vy, c->vz, c->temp, c->pr};
  memcpy(dst, d[which], sizeof(double) * (size_t)c->nx * c->nym * c->nzm);
}

static void explicit_terms(afid_cpu_t *c) {
  const int nxm = c->nxm, nym = c->nym, nzm = c->nzm;
  const double udy = c->dy * 0.25, udz = c->dz * 0.25, udyq = c->dyq / c->ren, udzq = c->dzq / c->ren;
  const double tudz = c->dz * 0.5, tudy = c->dy * 0.5, tudzq = c->dzq / c->pect, tudyq = c->dyq / c->pect;
  const double *vx = c->vx, *vy = c->vy, *vz = c->vz, *t = c->temp;
#pragma omp parallel for schedule(static)
  for (int col = 0; col < nym * nzm; ++col) {
    const int j = col % nym, i = col / nym;
    const int jp = wp(j, nym), jm = wm(j, nym), ip = wp(i, nzm), im = wm(i, nzm);
    const size_t C = IDX(c, 0, j, i), JP = IDX(c, 0, jp, i), JM = IDX(c, 0, jm, i), IP = IDX(c, 0, j, ip),
                 IM = IDX(c, 0, j, im), JMIP = IDX(c, 0, jm, ip), JPIM = IDX(c, 0, jp, im);
    /* ExplicitTermsVX.F90:42-127 */
    for (int k = 1; k < nxm; ++k) {
      const int km = k - 1, kp = k + 1;
      const double *idx = c->idx;
      double vxc = vx[C + k];
      double hxz = c->udx3c[k] * udz *
                   ((idx[km] * vz[IP + km] + idx[k] * vz[IP + k]) * (vx[IP + k] + vxc) -
                    (idx[km] * vz[C + km] + idx[k] * vz[C + k]) * (vxc + vx[IM + k]));
      double hxy = c->udx3c[k] * udy *
                   ((idx[km] * vy[JP + km] + idx[k] * vy[JP + k]) * (vx[JP + k] + vxc) -
                    (idx[km] * vy[C + km] + idx[k] * vy[C + k]) * (vxc + vx[JM + k]));
      double hxx = ((vx[C + kp] + vxc) * (vx[C + kp] + vxc) - (vxc + vx[C + km]) * (vxc + vx[C + km])) *
                   c->udx3c[k] * 0.25;
      double dzzvx = (vx[IM + k] - 2.0 * vxc + vx[IP + k]) * udzq;
      double dyyvx = (vx[JM + k] - 2.0 * vxc + vx[JP + k]) * udyq;
      double q = -(hxx + hxy + hxz) + dyyvx + dzzvx;
      if (c->gaxis == 1) q = q + c->byct * (c->active_t * 0.5 * (t[C + k] + t[C + km]));
      c->qcap[C + k] = q;
    }
    for (int k = 0; k < nxm; ++k) {
      const int kmm = k == 0 ? 0 : k - 1, kpp = k == nxm - 1 ? k : k + 1, kp = k + 1;
      /* ExplicitTermsVY.F90:44-122 */
      double cc = vy[C + k];
      double hyx = ((vx[C + kp] + vx[JM + kp]) * (vy[C + kpp] + cc) - (vx[C + k] + vx[JM + k]) * (cc + vy[C + kmm])) *
                   c->udx3m[k] * 0.25;
      double hyy = ((vy[JP + k] + cc) * (vy[JP + k] + cc) - (vy[JM + k] + cc) * (vy[JM + k] + cc)) * udy;
      double hyz = ((vy[IP + k] + cc) * (vz[IP + k] + vz[JMIP + k]) - (cc + vy[IM + k]) * (vz[C + k] + vz[JM + k])) * udz;
      double dyyvy = (vy[JP + k] - 2.0 * cc + vy[JM + k]) * udyq;
      double dzzvy = (vy[IP + k] - 2.0 * cc + vy[IM + k]) * udzq;
      double dph = -(hyx + hyy + hyz) + dyyvy + dzzvy + c->gy;
      if (c->gaxis == 2) dph = dph + c->byct * (c->active_t * 0.5 * (t[C + k] + t[JM + k]));
      c->dph[C + k] = dph;
      /* ExplicitTermsVZ.F90:38-118 */
      cc = vz[C + k];
      double hzz = ((vz[IP + k] + cc) * (vz[IP + k] + cc) - (vz[IM + k] + cc) * (vz[IM + k] + cc)) * udz;
      double hzy = ((vy[JP + k] + vy[JPIM + k]) * (vz[JP + k] + cc) - (vy[C + k] + vy[IM + k]) * (cc + vz[JM + k])) * udy;
      double hzx = ((vx[C + kp] + vx[IM + kp]) * (vz[C + kpp] + cc) - (vx[C + k] + vx[IM + k]) * (cc + vz[C + kmm])) *
                   c->udx3m[k] * 0.25;
      double dzzvz = (vz[IP + k] - 2.0 * cc + vz[IM + k]) * udzq;
      double dyyvz = (vz[JP + k] - 2.0 * cc + vz[JM + k]) * udyq;
      double dq = -(hzx + hzy + hzz) + dyyvz + dzzvz;
      if (c->gaxis == 3) dq = dq + c->byct * (c->active_t * 0.5 * (t[C + k] + t[IM + k]));
      c->dq[C + k] = dq;
      /* ExplicitTermsTemp.F90:34-77 */
      double tc = t[C + k], htx;
      const double tbp = c->tempbp[j + nym * i], ttp = c->temptp[j + nym * i];
      if (k == 0)
        htx = (vx[C + 1] * (t[C + 1] + tc) - vx[C] * 2.0 * tbp) * 0.5 * c->udx3m[0];
      else if (k == nxm - 1)
        htx = (vx[C + k + 1] * 2.0 * ttp - vx[C + k] * (tc + t[C + k - 1])) * 0.5 * c->udx3m[k];
      else
        htx = (vx[C + k + 1] * (t[C + k + 1] + tc) - vx[C + k] * (tc + t[C + k - 1])) * 0.5 * c->udx3m[k];
      double htz = (vz[IP + k] * (t[IP + k] + tc) - vz[C + k] * (tc + t[IM + k])) * tudz;
      double hty = (vy[JP + k] * (t[JP + k] + tc) - vy[C + k] * (tc + t[JM + k])) * tudy;
      double dzzt = (t[IP + k] - 2.0 * tc + t[IM + k]) * tudzq;
      double dyyt = (t[JP + k] - 2.0 * tc + t[JM + k]) * tudyq;
      c->hro[C + k] = -(htx + hty + htz) + dyyt + dzzt;
    }
  }
}

/* Normalised constant CN matrix rows (SolveImpEqnUpdate_*.F90) factored once with gttrf. */
typedef struct {
  int n;
  double *dl, *d, *du, *du2, *sc;
  int *ipiv;
} cnmat;

static void cn_build(cnmat *m, int n, int off, const double *am, const double *ac, const double *ap,
                     double betadx, int identity_ends) {
  m->n = n;
  m->dl = (double *)calloc(n, 8); m->d = (double *)calloc(n, 8); m->du = (double *)calloc(n, 8);
  m->du2 = (double *)calloc(n, 8); m->sc = (double *)calloc(n, 8); m->ipiv = (int *)calloc(n, sizeof(int));
  double *amkl = (double *)calloc(n, 8), *apkl = (double *)calloc(n, 8);
  for (int r = 0; r < n; ++r) {
    int k = r + off;
    if (identity_ends && (r == 0 || r == n - 1)) { amkl[r] = 0; apkl[r] = 0; m->d[r] = 1.0; m->sc[r] = 0.0; continue; }
    double b = 1.0 / (1.0 - ac[k] * betadx);
    amkl[r] = -am[k] * betadx * b;
    apkl[r] = -ap[k] * betadx * b;
    m->d[r] = 1.0;
    m->sc[r] = b;
  }
  for (int r = 0; r < n - 1; ++r) { m->dl[r] = amkl[r + 1]; m->du[r] = apkl[r]; }
  gttrf(n, m->dl, m->d, m->du, m->du2, m->ipiv);
  free(amkl); free(apkl);
}
static void cn_free(cnmat *m) { free(m->dl); free(m->d); free(m->du); free(m->du2); free(m->sc); free(m->ipiv); }

static void implicit_update(afid_cpu_t *c, double al, double ga, double ro, double dt, double beta) {
  const int nxm = c->nxm, nym = c->nym, nzm = c->nzm, nx = c->nx;
  cnmat mx, my, mt;
  cn_build(&mx, nx, 0, c->am3ck, c->ac3ck, c->ap3ck, beta * al, 1);
  cn_build(&my, nxm, 0, c->am3sk, c->ac3sk, c->ap3sk, beta * al, 0);
  cn_build(&mt, nxm, 0, c->am3ssk, c->ac3ssk, c->ap3ssk, 0.5 * al * dt / c->pect, 0);
  const double alre = al / c->ren, alpec = al / c->pect, udyp = c->dy * al;
#pragma omp parallel
  {
    double *rhs = (double *)malloc(sizeof(double) * (nx + 1));
#pragma omp for schedule(static)
    for (int col = 0; col < nym * nzm; ++col) {
      const int j = col % nym, i = col / nym, jm = wm(j, nym), im = wm(i, nzm);
      const size_t C = IDX(c, 0, j, i), JM = IDX(c, 0, jm, i), IM = IDX(c, 0, j, im);
      double *vx = c->vx, *vy = c->vy, *vz = c->vz, *t = c->temp, *pr = c->pr;
      /* ImplicitAndUpdateVX.F90:37-87 */
      rhs[0] = 0.0; rhs[nx - 1] = 0.0;
      for (int k = 1; k < nxm; ++k) {
        double dxx = vx[C + k + 1] * c->ap3ck[k] + vx[C + k] * c->ac3ck[k] + vx[C + k - 1] * c->am3ck[k];
        double dxp = (pr[C + k] - pr[C + k - 1]) * (al * c->udx3c[k]);
        rhs[k] = (ga * c->qcap[C + k] + ro * c->rux[C + k] + alre * dxx - dxp) * dt * mx.sc[k];
        c->rux[C + k] = c->qcap[C + k];
      }
      gttrs_r(nx, mx.dl, mx.d, mx.du, mx.du2, mx.ipiv, rhs);
      for (int k = 1; k < nxm; ++k) vx[C + k] += rhs[k];
      vx[C] = 0.0; vx[C + nx - 1] = 0.0;
      /* ImplicitAndUpdateVY.F90:40-93 */
      for (int k = 0; k < nxm; ++k) {
        const int kmm = k == 0 ? 0 : k - 1, kpp = k == nxm - 1 ? k : k + 1;
        double amm = c->am3sk[k], acc = c->ac3sk[k], app = c->ap3sk[k], dxx;
        if (k == 0) dxx = vy[C + kpp] * app + vy[C + k] * acc - (acc + app) * c->xminusu * c->inslws;
        else if (k == nxm - 1) dxx = -(acc + amm) * c->xplusu * c->inslwn + vy[C + k] * acc + vy[C + kmm] * amm;
        else dxx = vy[C + kpp] * app + vy[C + k] * acc + vy[C + kmm] * amm;
        double dyp = (pr[C + k] - pr[JM + k]) * udyp;
        rhs[k] = (ga * c->dph[C + k] + ro * c->ruy[C + k] + alre * dxx - dyp) * dt * my.sc[k];
        c->ruy[C + k] = c->dph[C + k];
      }
      gttrs_r(nxm, my.dl, my.d, my.du, my.du2, my.ipiv, rhs);
      for (int k = 0; k < nxm; ++k) vy[C + k] += rhs[k];
      /* ImplicitAndUpdateVZ.F90:38-77 */
      for (int k = 0; k < nxm; ++k) {
        const int kmm = k == 0 ? 0 : k - 1, kpp = k == nxm - 1 ? k : k + 1;
        double dxx = vz[C + kpp] * c->ap3sk[k] + vz[C + k] * c->ac3sk[k] + vz[C + kmm] * c->am3sk[k];
        double dzp = (pr[C + k] - pr[IM + k]) * c->dz * al;
        rhs[k] = (ga * c->dq[C + k] + ro * c->ruz[C + k] + alre * dxx - dzp) * dt * my.sc[k];
        c->ruz[C + k] = c->dq[C + k];
      }
      gttrs_r(nxm, my.dl, my.d, my.du, my.du2, my.ipiv, rhs);
      for (int k = 0; k < nxm; ++k) vz[C + k] += rhs[k];
      /* ImplicitAndUpdateTemp.F90:33-74 */
      const double tbp = c->tempbp[j + nym * i], ttp = c->temptp[j + nym * i];
      for (int k = 0; k < nxm; ++k) {
        double dxx;
        if (k == 0) dxx = t[C + 1] * c->ap3ssk[0] + t[C] * c->ac3ssk[0] - (c->ap3ssk[0] + c->ac3ssk[0]) * tbp * c->tfixs;
        else if (k == nxm - 1)
          dxx = t[C + k] * c->ac3ssk[k] + t[C + k - 1] * c->am3ssk[k] - (c->am3ssk[k] + c->ac3ssk[k]) * ttp * c->tfixn;
        else dxx = t[C + k + 1] * c->ap3ssk[k] + t[C + k] * c->ac3ssk[k] + t[C + k - 1] * c->am3ssk[k];
        rhs[k] = (ga * c->hro[C + k] + ro * c->rut[C + k] + alpec * dxx) * dt * mt.sc[k];
        c->rut[C + k] = c->hro[C + k];
      }
      gttrs_r(nxm, mt.dl, mt.d, mt.du, mt.du2, mt.ipiv, rhs);
      for (int k = 0; k < nxm; ++k) t[C + k] += rhs[k];
    }
    free(rhs);
  }
  cn_free(&mx); cn_free(&my); cn_free(&mt);
}

static void pressure(afid_cpu_t *c, double al, double dt, double beta) {
  const int nxm = c->nxm, nym = c->nym, nzm = c->nzm, nyh = nym / 2 + 1;
  const double usdtal = 1.0 / (dt * al);
  cplx *sp = c->spec;
  /* CalcLocalDivergence (pressure.F90:149-161) + y r2c FFT per (i, k) line (pressure.F90:174) */
#pragma omp parallel
  {
    cplx *a = (cplx *)malloc(sizeof(cplx) * nym), *w = (cplx *)malloc(sizeof(cplx) * nym);
#pragma omp for schedule(static)
    for (int line = 0; line < nzm * nxm; ++line) {
      const int i = line / nxm, k = line % nxm, ip = wp(i, nzm);
      for (int j = 0; j < nym; ++j) {
        const int jp = wp(j, nym);
        double dq = (c->vz[IDX(c, k, j, ip)] - c->vz[IDX(c, k, j, i)]) * c->dz +
                    (c->vy[IDX(c, k, jp, i)] - c->vy[IDX(c, k, j, i)]) * c->dy +
                    (c->vx[IDX(c, k + 1, j, i)] - c->vx[IDX(c, k, j, i)]) * c->udx3m[k];
        a[j] = dq * usdtal;
      }
      fft1(a, w, nym, c->fy, c->nfy, c->twy, 0);
      for (int ky = 0; ky < nyh; ++ky) sp[(size_t)k + (size_t)nxm * (ky + (size_t)nyh * i)] = a[ky];
    }
    free(a); free(w);
  }
  /* z c2c FFT, scale 1/(nym*nzm) (pressure.F90:176-179), tridiagonal per mode (:201-236),
     backward z FFT (:189) */
#pragma omp parallel
  {
    cplx *a = (cplx *)malloc(sizeof(cplx) * nzm), *w = (cplx *)malloc(sizeof(cplx) * nzm);
#pragma omp for schedule(static)
    for (int line = 0; line < nyh * nxm; ++line) {
      const int ky = line / nxm, k = line % nxm;
      for (int i = 0; i < nzm; ++i) a[i] = sp[(size_t)k + (size_t)nxm * (ky + (size_t)nyh * i)];
      fft1(a, w, nzm, c->fz, c->nfz, c->twz, 0);
      for (int i = 0; i < nzm; ++i) sp[(size_t)k + (size_t)nxm * (ky + (size_t)nyh * i)] = a[i] / (double)(nzm * nym);
    }
    free(a); free(w);
  }
#pragma omp parallel
  {
    double *dl = (double *)malloc(8 * nxm), *d = (double *)malloc(8 * nxm), *du = (double *)malloc(8 * nxm),
           *du2 = (double *)malloc(8 * nxm);
    int *ipiv = (int *)malloc(sizeof(int) * nxm);
    cplx *b = (cplx *)malloc(sizeof(cplx) * nxm);
#pragma omp for schedule(static)
    for (int mode = 0; mode < nyh * nzm; ++mode) {
      const int ky = mode % nyh, kz = mode / nyh;
      cplx *col = sp + (size_t)nxm * (ky + (size_t)nyh * kz);
      for (int k = 0; k < nxm; ++k) {
        double f = 1.0 / (c->acphk[k] - c->ak2[ky] - c->ak1[kz]);
        b[k] = col[k] * f;
        if (k < nxm - 1) du[k] = c->apphk[k] * f;
        if (k > 0) dl[k - 1] = c->amphk[k] * f;
        d[k] = 1.0 + 1.0e-15;
      }
      gttrf(nxm, dl, d, du, du2, ipiv);
      gttrs_c(nxm, dl, d, du, du2, ipiv, b);
      memcpy(col, b, sizeof(cplx) * nxm);
    }
    free(dl); free(d); free(du); free(du2); free(ipiv); free(b);
  }
#pragma omp parallel
  {
    cplx *a = (cplx *)malloc(sizeof(cplx) * nzm), *w = (cplx *)malloc(sizeof(cplx) * nzm);
#pragma omp for schedule(static)
    for (int line = 0; line < nyh * nxm; ++line) {
      const int ky = line / nxm, k = line % nxm;
      for (int i = 0; i < nzm; ++i) a[i] = sp[(size_t)k + (size_t)nxm * (ky + (size_t)nyh * i)];
      fft1(a, w, nzm, c->fz, c->nfz, c->twz, 1);
      for (int i = 0; i < nzm; ++i) sp[(size_t)k + (size_t)nxm * (ky + (size_t)nyh * i)] = a[i];
    }
    free(a); free(w);
  }
  /* y c2r (pressure.F90:193): Hermitian extension, imaginary DC/Nyquist ignored */
#pragma omp parallel
  {
    cplx *a = (cplx *)malloc(sizeof(cplx) * nym), *w = (cplx *)malloc(sizeof(cplx) * nym);
#pragma omp for schedule(static)
    for (int line = 0; line < nzm * nxm; ++line) {
      const int i = line / nxm, k = line % nxm;
      for (int j = 0; j < nym; ++j) {
        int jj = (2 * j > nym) ? nym - j : j;
        cplx v = sp[(size_t)k + (size_t)nxm * (jj + (size_t)nyh * i)];
        if (jj == 0 || 2 * jj == nym) v = creal(v);
        a[j] = (2 * j > nym) ? conj(v) : v;
      }
      fft1(a, w, nym, c->fy, c->nfy, c->twy, 1);
      for (int j = 0; j < nym; ++j) c->phi[IDX(c, k, j, i)] = creal(a[j]);
    }
    free(a); free(w);
  }
  /* RemoveDivergence (pressure.F90:245-266) and CorrectPressure (:276-300) */
  const double udy = al * dt * c->dy, udz = al * dt * c->dz, be = al * beta;
  const double *ph = c->phi;
#pragma omp parallel for schedule(static)
  for (int col = 0; col < nym * nzm; ++col) {
    const int j = col % nym, i = col / nym, jm = wm(j, nym), jp = wp(j, nym), im = wm(i, nzm), ip = wp(i, nzm);
    const size_t C = IDX(c, 0, j, i), JM = IDX(c, 0, jm, i), JP = IDX(c, 0, jp, i), IM = IDX(c, 0, j, im),
                 IP = IDX(c, 0, j, ip);
    for (int k = 0; k < nxm; ++k) {
      const int km = k == 0 ? 0 : k - 1, kp = k == nxm - 1 ? k : k + 1;
      const double usukm = al * dt * c->udx3c[k], l = ph[C + k];
      c->vx[C + k] = c->vx[C + k] - (l - ph[C + km]) * usukm;
      c->vy[C + k] = c->vy[C + k] - (l - ph[JM + k]) * udy;
      c->vz[C + k] = c->vz[C + k] - (l - ph[IM + k]) * udz;
      c->pr[C + k] = c->pr[C + k] + l -
                     be * ((ph[IP + k] - 2.0 * l + ph[IM + k]) * c->dzq + (ph[JP + k] - 2.0 * l + ph[JM + k]) * c->dyq +
                           (ph[C + kp] * c->apphk[k] + l * c->acphk[k] + ph[C + km] * c->amphk[k]));
    }
  }
}

/* TimeMarcher.F90:28-133 */
void afid_cpu_timemarcher(afid_cpu_t *c, double dt) {
  double gam[3], rom[3];
  if (c->nsst > 1) { gam[0] = 8.0 / 15.0; gam[1] = 5.0 / 12.0; gam[2] = 3.0 / 4.0; rom[0] = 0.0; rom[1] = -17.0 / 60.0; rom[2] = -5.0 / 12.0; }
  else { gam[0] = 1.5; gam[1] = 0.0; gam[2] = 0.0; rom[0] = -0.5; rom[1] = 0.0; rom[2] = 0.0; }
  const double beta = dt / c->ren * 0.5;
  const int ns_n = c->nsst > 1 ? 3 : 1;
  for (int ns = 0; ns < ns_n; ++ns) {
    const double al = gam[ns] + rom[ns];
    explicit_terms(c);
    implicit_update(c, al, gam[ns], rom[ns], dt, beta);
    pressure(c, al, dt, beta);
  }
}

/* CalcMaxCFL.F90:22-43 */
double afid_cpu_cfl(const afid_cpu_t *c) {
  const int nxm = c->nxm, nym = c->nym, nzm = c->nzm;
  double m = 0.00000001;
#pragma omp parallel for reduction(max : m) schedule(static)
  for (int col = 0; col < nym * nzm; ++col) {
    const int j = col % nym, i = col / nym, jp = wp(j, nym), ip = wp(i, nzm);
    for (int k = 0; k < nxm; ++k) {
      double q = fabs((c->vz[IDX(c, k, j, i)] + c->vz[IDX(c, k, j, ip)]) * 0.5 * c->dz) +
                 fabs((c->vy[IDX(c, k, j, i)] + c->vy[IDX(c, k, jp, i)]) * 0.5 * c->dy) +
                 fabs((c->vx[IDX(c, k, j, i)] + c->vx[IDX(c, k + 1, j, i)]) * 0.5 * c->udx3m[k]);
      if (q > m) m = q;
    }
  }
  return m;
}

/* GlobalQuantities.F90:35-79, 87-91 and the first and last rows of CalcMeanProfiles' Tbar
 * (CalcMeanProfiles.F90:48-50, 88): out = {Nu_vol, kinetic energy 0.5 <|u|^2> (g3rc-weighted),
 * Tbar(1), Tbar(nxm)}; ra_pr = Pr*|Ra|.  Column sums are accumulated in column order. */
void afid_cpu_stats(const afid_cpu_t *c, double ra_pr, double *out) {
  const int nxm = c->nxm, nym = c->nym, nzm = c->nzm, ncol = nym * nzm;
  double *part = (double *)calloc((size_t)ncol * 4, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int col = 0; col < ncol; ++col) {
    const int j = col % nym, i = col / nym;
    double anu = 0.0, ke = 0.0;
    for (int k = 0; k < nxm; ++k) {
      const size_t q = IDX(c, k, j, i);
      const double fac2 = c->g3rc[k];
      anu += c->temp[q] * ((c->vx[q] + c->vx[q + 1]) * 0.5) * fac2;
      ke += fac2 * (c->vz[q] * c->vz[q] + c->vy[q] * c->vy[q] + c->vx[q] * c->vx[q]);
    }
    part[4 * col + 0] = anu;
    part[4 * col + 1] = ke;
    part[4 * col + 2] = c->temp[IDX(c, 0, j, i)];
    part[4 * col + 3] = c->temp[IDX(c, nxm - 1, j, i)];
  }
  double sum[4] = {0.0, 0.0, 0.0, 0.0};
  for (int col = 0; col < ncol; ++col)
    for (int q = 0; q < 4; ++q) sum[q] += part[4 * col + q];
  free(part);
  const double vol = 1.0 / ((double)nxm * (double)nzm * (double)nym);  /* alx3 * dx = nxm */
  out[0] = 1.0 + sqrt(ra_pr) * sum[0] * vol;
  out[1] = 0.5 * sum[1] * vol;
  out[2] = sum[2] / ((double)nym * (double)nzm);
  out[3] = sum[3] / ((double)nym * (double)nzm);
}

/* ============================================================================================
 * Multi-resolution salinity (salinity.F90, multires/InterpVelMgrd.F90, HermiteInterpolations.F90):
 * the same routines as oracle/afid_salinity.py, on the per-target stencils of afid_mgrd_create
 * (first source row + 4 weights per target; x sources are wall-extended columns with rows
 * -2 .. n+1, y/z sources wrap).  Refined fields are x fastest with stride nxr = nxmr + 1.
 * ============================================================================================ */
typedef struct {
  afid_cpu_t *c;
  int nxmr, nymr, nzmr, nxr, sfixs, sfixn, active_s;
  double dxr, dyr, dzr, pecs, bycs;
  double *lxa, *udx3mr, *tdxr, *ap, *ac, *am, *salbp, *saltp;
  int *st[6];
  double *w[6];
  double *sal, *rusal, *vxr, *vyr, *vzr, *salc, *hsal;
  double *tz;   /* z-contracted coarse gradients, 3 x nx*nym*nzmr */
  double *u;    /* z-contracted extended refined salinity, (nxmr+4) * nymr * nzm */
  double *gyr, *gzr;
} afid_cpu_sal_t;

static int wrapi(int a, int n) { a %= n; return a < 0 ? a + n : a; }

/* tab: xcr[nxmr+1], udx3mr, g3rmr, ap3sskr, ac3sskr, am3sskr [nxmr], salbp, saltp [nymr*nzmr];
   dprm: dxr dyr dzr pecs bycs; iprm: nxmr nymr nzmr active_s sfixs sfixn;
   st/w: to_ref x y z, to_coarse x y z (sizes nxmr nymr nzmr nxm nym nzm). */
afid_cpu_sal_t *afid_cpu_sal_create(afid_cpu_t *c, const double *tab[8], const double *dprm, const int *iprm,
                                    const int *st[6], const double *w[6]) {
  afid_cpu_sal_t *s = (afid_cpu_sal_t *)calloc(1, sizeof(afid_cpu_sal_t));
  s->c = c;
  s->nxmr = iprm[0]; s->nymr = iprm[1]; s->nzmr = iprm[2]; s->active_s = iprm[3]; s->sfixs = iprm[4]; s->sfixn = iprm[5];
  s->nxr = s->nxmr + 1;
  s->dxr = dprm[0]; s->dyr = dprm[1]; s->dzr = dprm[2]; s->pecs = dprm[3]; s->bycs = dprm[4];
  const int n = s->nxmr, npl = s->nymr * s->nzmr;
  s->lxa = (double *)malloc(8 * n); s->tdxr = (double *)malloc(8 * n);
  for (int k = 0; k < n; ++k) { s->lxa[k] = tab[0][k + 1] - tab[0][k]; s->tdxr[k] = 0.5 * s->dxr / tab[2][k]; }
  s->udx3mr = dup(tab[1], n); s->ap = dup(tab[3], n); s->ac = dup(tab[4], n); s->am = dup(tab[5], n);
  s->salbp = dup(tab[6], npl); s->saltp = dup(tab[7], npl);
  const int sizes[6] = {n, s->nymr, s->nzmr, c->nxm, c->nym, c->nzm};
  for (int d = 0; d < 6; ++d) {
    s->st[d] = (int *)malloc(sizeof(int) * sizes[d]);
    memcpy(s->st[d], st[d], sizeof(int) * sizes[d]);
    s->w[d] = dup(w[d], 4 * sizes[d]);
  }
  const size_t nr = (size_t)s->nxr * npl, ncs = (size_t)c->nx * c->nym * c->nzm;
  double **f[] = {&s->sal, &s->rusal, &s->vxr, &s->vyr, &s->vzr, &s->hsal, &s->gyr, &s->gzr};
  for (size_t q = 0; q < sizeof f / sizeof f[0]; ++q) *f[q] = (double *)calloc(nr, 8);
  s->salc = (double *)calloc(ncs, 8);
  s->tz = (double *)calloc(3 * (size_t)c->nx * c->nym * s->nzmr, 8);
  s->u = (double *)calloc((size_t)(n + 4) * s->nymr * c->nzm, 8);
  return s;
}

void afid_cpu_sal_destroy(afid_cpu_sal_t *s) {
  if (!s) return;
  double *a[] = {s->lxa, s->tdxr, s->udx3mr, s->ap, s->ac, s->am, s->salbp, s->saltp, s->sal, s->rusal, s->vxr,
                 s->vyr, s->vzr, s->hsal, s->gyr, s->gzr, s->salc, s->tz, s->u};
  for (size_t q = 0; q < sizeof a / sizeof a[0]; ++q) free(a[q]);
  for (int d = 0; d < 6; ++d) { free(s->st[d]); free(s->w[d]); }
  free(s);
}

static size_t RIDX(const afid_cpu_sal_t *s, int k, int j, int i) { return (size_t)k + (size_t)s->nxr * ((size_t)j + (size_t)s->nymr * i); }

/* wall-extended coarse row r of a column (InterpVelMgrd.F90:40-41) */
static double cext(const double *col, int r, int nxm, double fs, double fn) {
  if (r >= 0 && r < nxm) return col[r];
  if (r == -1) return fs * col[0];
  if (r == nxm) return fn * col[nxm - 1];
  return 0.0;
}
/* wall-extended refined salinity row r (salinity.F90:462-481) */
static double sext(const afid_cpu_sal_t *s, const double *col, int r, int pl) {
  const int n = s->nxmr;
  if (r >= 0 && r < n) return col[r];
  if (r == -1) return s->sfixs ? 2.0 * s->salbp[pl] - col[0] : col[0];
  if (r == n) return s->sfixn ? 2.0 * s->saltp[pl] - col[n - 1] : col[n - 1];
  return 0.0;
}

/* InterpVelMgrd (one rank) */
static void sal_interp_vel(afid_cpu_sal_t *s) {
  afid_cpu_t *c = s->c;
  const int nxm = c->nxm, nym = c->nym, nzm = c->nzm, nx = c->nx;
  const double fs = (double)(1 - 2 * c->inslws), fn = (double)(1 - 2 * c->inslwn);
  const size_t nt = (size_t)nx * nym * s->nzmr;
  /* gradients at the coarse centres, contracted in z (z first) */
#pragma omp parallel for schedule(static)
  for (int col = 0; col < nym * s->nzmr; ++col) {
    const int jc = col % nym, ir = col / nym;
    const int sz = s->st[2][ir];
    const double *wz = s->w[2] + 4 * ir;
    for (int r = 0; r < nxm; ++r) {
      double t[3];
      for (int cc = 0; cc < 4; ++cc) {
        const int ic = wrapi(sz + cc, nzm);
        const size_t e = IDX(c, r, jc, ic);
        const double gx = (c->vx[e + 1] - c->vx[e]) * c->udx3m[r];
        const double gy = (c->vy[IDX(c, r, wp(jc, nym), ic)] - c->vy[e]) * c->dy;
        const double gz = (c->vz[IDX(c, r, jc, wp(ic, nzm))] - c->vz[e]) * c->dz;
        if (cc == 0) { t[0] = gx * wz[0]; t[1] = gy * wz[0]; t[2] = gz * wz[0]; }
        else { t[0] += gx * wz[cc]; t[1] += gy * wz[cc]; t[2] += gz * wz[cc]; }
      }
      const size_t o = (size_t)r + (size_t)nx * ((size_t)jc + (size_t)nym * ir);
      s->tz[o] = t[0]; s->tz[nt + o] = t[1]; s->tz[2 * nt + o] = t[2];
    }
  }
  /* y then x per refined column; vxr integrated along x (InterpVelMgrd.F90:48-57) */
#pragma omp parallel
  {
    double *q = (double *)malloc(sizeof(double) * 3 * (nxm + 4));
#pragma omp for schedule(static)
    for (int col = 0; col < s->nymr * s->nzmr; ++col) {
      const int jr = col % s->nymr, ir = col / s->nymr;
      const int sy = s->st[1][jr];
      const double *wy = s->w[1] + 4 * jr;
      for (int f = 0; f < 3; ++f) {
        double *qf = q + f * (nxm + 4);
        for (int r = 0; r < nxm; ++r) {
          double v = 0.0;
          for (int b = 0; b < 4; ++b) {
            const size_t o = (size_t)r + (size_t)nx * ((size_t)wrapi(sy + b, nym) + (size_t)nym * ir);
            v = (b == 0) ? s->tz[f * nt + o] * wy[0] : v + s->tz[f * nt + o] * wy[b];
          }
          qf[r + 2] = v;
        }
        qf[0] = 0.0; qf[1] = fs * qf[2]; qf[nxm + 2] = fn * qf[nxm + 1]; qf[nxm + 3] = 0.0;
      }
      const size_t R = RIDX(s, 0, jr, ir);
      s->vxr[R] = 0.0;
      for (int kr = 0; kr < s->nxmr; ++kr) {
        const int p = s->st[0][kr] + 2;
        const double *wx = s->w[0] + 4 * kr;
        double g[3];
        for (int f = 0; f < 3; ++f) {
          const double *qf = q + f * (nxm + 4);
          g[f] = qf[p] * wx[0] + qf[p + 1] * wx[1] + qf[p + 2] * wx[2] + qf[p + 3] * wx[3];
        }
        s->vxr[R + kr + 1] = s->vxr[R + kr] + g[0] * s->lxa[kr];
        s->gyr[R + kr] = g[1];
        s->gzr[R + kr] = g[2];
      }
    }
    free(q);
  }
  /* vyr: first guess at y = 0 (z, then x), integrated along y (:99-131) */
  const double lya = 1. / s->dyr, lza = 1. / s->dzr;
#pragma omp parallel for schedule(static)
  for (int ir = 0; ir < s->nzmr; ++ir) {
    const int sz = s->st[2][ir];
    const double *wz = s->w[2] + 4 * ir;
    for (int kr = 0; kr < s->nxmr; ++kr) {
      const int sx = s->st[0][kr];
      const double *wx = s->w[0] + 4 * kr;
      double v = 0.0;
      for (int a = 0; a < 4; ++a) {
        double q1 = 0.0;
        for (int cc = 0; cc < 4; ++cc) {
          const double e = cext(c->vy + IDX(c, 0, 0, wrapi(sz + cc, nzm)), sx + a, nxm, fs, fn) * wz[cc];
          q1 = (cc == 0) ? e : q1 + e;
        }
        v = (a == 0) ? q1 * wx[a] : v + q1 * wx[a];
      }
      s->vyr[RIDX(s, kr, 0, ir)] = v;
      for (int jr = 0; jr + 1 < s->nymr; ++jr) {
        v = v + s->gyr[RIDX(s, kr, jr, ir)] * lya;
        s->vyr[RIDX(s, kr, jr + 1, ir)] = v;
      }
    }
  }
  /* vzr: first guess at z = 0 when nzm > 1 (y, then x), integrated along z (:181-213) */
#pragma omp parallel for schedule(static)
  for (int jr = 0; jr < s->nymr; ++jr) {
    const int sy = s->st[1][jr];
    const double *wy = s->w[1] + 4 * jr;
    for (int kr = 0; kr < s->nxmr; ++kr) {
      const int sx = s->st[0][kr];
      const double *wx = s->w[0] + 4 * kr;
      double v = 0.0;
      if (nzm > 1)
        for (int a = 0; a < 4; ++a) {
          double q1 = 0.0;
          for (int b = 0; b < 4; ++b) {
            const double e = cext(c->vz + IDX(c, 0, wrapi(sy + b, nym), 0), sx + a, nxm, fs, fn) * wy[b];
            q1 = (b == 0) ? e : q1 + e;
          }
          v = (a == 0) ? q1 * wx[a] : v + q1 * wx[a];
        }
      s->vzr[RIDX(s, kr, jr, 0)] = v;
      for (int ir = 0; ir + 1 < s->nzmr; ++ir) {
        v = v + s->gzr[RIDX(s, kr, jr, ir)] * lza;
        s->vzr[RIDX(s, kr, jr, ir + 1)] = v;
      }
    }
  }
}

/* InterpSalMultigrid: z, then y, then x on the wall-extended refined salinity */
static void sal_interp_sal(afid_cpu_sal_t *s) {
  afid_cpu_t *c = s->c;
  const int nxm = c->nxm, nym = c->nym, nzm = c->nzm, n = s->nxmr, L = n + 4;
#pragma omp parallel for schedule(static)
  for (int col = 0; col < s->nymr * nzm; ++col) {
    const int jr = col % s->nymr, ic = col / s->nymr;
    const int sz = s->st[5][ic];
    const double *wz = s->w[5] + 4 * ic;
    double *uo = s->u + (size_t)L * col;
    for (int q = 0; q < L; ++q) {
      double v = 0.0;
      for (int cc = 0; cc < 4; ++cc) {
        const int ir = wrapi(sz + cc, s->nzmr), pl = jr + s->nymr * ir;
        const double e = sext(s, s->sal + RIDX(s, 0, jr, ir), q - 2, pl) * wz[cc];
        v = (cc == 0) ? e : v + e;
      }
      uo[q] = v;
    }
  }
#pragma omp parallel
  {
    double *q2 = (double *)malloc(sizeof(double) * L);
#pragma omp for schedule(static)
    for (int col = 0; col < nym * nzm; ++col) {
      const int j = col % nym, i = col / nym;
      const int sy = s->st[4][j];
      const double *wy = s->w[4] + 4 * j;
      for (int q = 0; q < L; ++q) {
        double v = 0.0;
        for (int b = 0; b < 4; ++b) {
          const double e = s->u[(size_t)L * (wrapi(sy + b, s->nymr) + (size_t)s->nymr * i) + q] * wy[b];
          v = (b == 0) ? e : v + e;
        }
        q2[q] = v;
      }
      for (int k = 0; k < nxm; ++k) {
        const int p = s->st[3][k] + 2;
        const double *wx = s->w[3] + 4 * k;
        s->salc[IDX(c, k, j, i)] = q2[p] * wx[0] + q2[p + 1] * wx[1] + q2[p + 2] * wx[2] + q2[p + 3] * wx[3];
      }
    }
    free(q2);
  }
}

/* ExplicitSalinity + ImplicitSalinity + SolveImpEqnUpdate_Sal (salinity.F90:268-453) */
static void sal_step(afid_cpu_sal_t *s, double al, double ga, double ro, double dt) {
  const int n = s->nxmr, nymr = s->nymr, nzmr = s->nzmr;
  const double udyr = 0.5 * s->dyr, udzr = 0.5 * s->dzr, udyrq = s->dyr * s->dyr / s->pecs,
               udzrq = s->dzr * s->dzr / s->pecs, alpec = al / s->pecs;
  const double *sal = s->sal, *vxr = s->vxr, *vyr = s->vyr, *vzr = s->vzr;
  /* explicit terms from the old salinity into hsal, then the per-column update */
#pragma omp parallel for schedule(static)
  for (int col = 0; col < nymr * nzmr; ++col) {
    const int j = col % nymr, i = col / nymr;
    const size_t C = RIDX(s, 0, j, i), JP = RIDX(s, 0, wp(j, nymr), i), JM = RIDX(s, 0, wm(j, nymr), i),
                 IP = RIDX(s, 0, j, wp(i, nzmr)), IM = RIDX(s, 0, j, wm(i, nzmr));
    const double bp = s->salbp[col], tp = s->saltp[col];
    for (int k = 0; k < n; ++k) {
      const double sc = sal[C + k];
      double hsx;
      if (k == 0) hsx = (vxr[C + 1] * (sal[C + 1] + sc) - vxr[C] * 2.0 * bp) * s->udx3mr[k] * 0.5;
      else if (k == n - 1) hsx = (vxr[C + k + 1] * 2.0 * tp - vxr[C + k] * (sc + sal[C + k - 1])) * s->udx3mr[k] * 0.5;
      else hsx = (vxr[C + k + 1] * (sal[C + k + 1] + sc) - vxr[C + k] * (sc + sal[C + k - 1])) * s->udx3mr[k] * 0.5;
      const double hsy = (vyr[JP + k] * (sal[JP + k] + sc) - vyr[C + k] * (sc + sal[JM + k])) * udyr;
      const double hsz = (vzr[IP + k] * (sal[IP + k] + sc) - vzr[C + k] * (sc + sal[IM + k])) * udzr;
      const double dyys = (sal[JP + k] - 2.0 * sc + sal[JM + k]) * udyrq;
      const double dzzs = (sal[IP + k] - 2.0 * sc + sal[IM + k]) * udzrq;
      s->hsal[C + k] = -(hsx + hsy + hsz) + dyys + dzzs;
    }
  }
  cnmat ms;
  cn_build(&ms, n, 0, s->am, s->ac, s->ap, 0.5 * al * dt / s->pecs, 0);
#pragma omp parallel
  {
    double *rhs = (double *)malloc(sizeof(double) * (n + 1));
#pragma omp for schedule(static)
    for (int col = 0; col < nymr * nzmr; ++col) {
      const size_t C = RIDX(s, 0, col % nymr, col / nymr);
      const double bp = s->salbp[col], tp = s->saltp[col];
      double *sl = s->sal + C;
      for (int k = 0; k < n; ++k) {
        double dxx;
        if (k == 0) dxx = sl[1] * s->ap[0] + sl[0] * s->ac[0] - (s->ap[0] + s->ac[0]) * bp * s->sfixs;
        else if (k == n - 1) dxx = sl[k] * s->ac[k] + sl[k - 1] * s->am[k] - (s->am[k] + s->ac[k]) * tp * s->sfixn;
        else dxx = sl[k + 1] * s->ap[k] + sl[k] * s->ac[k] + sl[k - 1] * s->am[k];
        rhs[k] = (ga * s->hsal[C + k] + ro * s->rusal[C + k] + alpec * dxx) * dt * ms.sc[k];
        s->rusal[C + k] = s->hsal[C + k];
      }
      gttrs_r(n, ms.dl, ms.d, ms.du, ms.du2, ms.ipiv, rhs);
      for (int k = 0; k < n; ++k) sl[k] += rhs[k];
    }
    free(rhs);
  }
  cn_free(&ms);
}

void afid_cpu_sal_set(afid_cpu_sal_t *s, const double *sal) {
  memcpy(s->sal, sal, sizeof(double) * (size_t)s->nxr * s->nymr * s->nzmr);
  memset(s->rusal, 0, sizeof(double) * (size_t)s->nxr * s->nymr * s->nzmr);
  sal_interp_vel(s);
  sal_interp_sal(s);
}
void afid_cpu_sal_get(const afid_cpu_sal_t *s, double *sal) {
  memcpy(sal, s->sal, sizeof(double) * (size_t)s->nxr * s->nymr * s->nzmr);
}

/* TimeMarcher.F90:28-150 with salinity */
void afid_cpu_timemarcher_sal(afid_cpu_sal_t *s, double dt) {
  afid_cpu_t *c = s->c;
  double gam[3], rom[3];
  if (c->nsst > 1) { gam[0] = 8.0 / 15.0; gam[1] = 5.0 / 12.0; gam[2] = 3.0 / 4.0; rom[0] = 0.0; rom[1] = -17.0 / 60.0; rom[2] = -5.0 / 12.0; }
  else { gam[0] = 1.5; gam[1] = 0.0; gam[2] = 0.0; rom[0] = -0.5; rom[1] = 0.0; rom[2] = 0.0; }
  const double beta = dt / c->ren * 0.5;
  const int ns_n = c->nsst > 1 ? 3 : 1;
  const size_t nc = (size_t)c->nx * c->nym * c->nzm;
  for (int ns = 0; ns < ns_n; ++ns) {
    const double al = gam[ns] + rom[ns];
    explicit_terms(c);
    if (s->active_s == 1) { /* AddSalBuoyancy (salinity.F90:494-506) */
      double *tgt = c->gaxis == 1 ? c->qcap : (c->gaxis == 2 ? c->dph : c->dq);
#pragma omp parallel for schedule(static)
      for (size_t e = 0; e < nc; ++e)
        if ((int)(e % c->nx) < c->nxm) tgt[e] = tgt[e] - s->bycs * s->salc[e];
    }
    sal_step(s, al, gam[ns], rom[ns], dt);
    implicit_update(c, al, gam[ns], rom[ns], dt, beta);
    pressure(c, al, dt, beta);
    sal_interp_vel(s);
    sal_interp_sal(s);
  }
}

/* CalcMaxCFL.F90:48-65 (refined grid) */
double afid_cpu_sal_cfl(const afid_cpu_sal_t *s) {
  double m = 1.0e-8;
#pragma omp parallel for reduction(max : m) schedule(static)
  for (int col = 0; col < s->nymr * s->nzmr; ++col) {
    const int j = col % s->nymr, i = col / s->nymr;
    const size_t C = RIDX(s, 0, j, i), JP = RIDX(s, 0, wp(j, s->nymr), i), IP = RIDX(s, 0, j, wp(i, s->nzmr));
    for (int k = 0; k < s->nxmr; ++k) {
      const double q = fabs((s->vzr[C + k] + s->vzr[IP + k]) * 0.5 * s->dzr) +
                       fabs((s->vyr[C + k] + s->vyr[JP + k]) * 0.5 * s->dyr) +
                       fabs((s->vxr[C + k] + s->vxr[C + k + 1]) * 0.5 * s->udx3mr[k]);
      if (q > m) m = q;
    }
  }
  return m;
}
