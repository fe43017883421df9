// afid_api.cu — the C ABI of include/afid_gpu.h: context lifetime, state transfer, and the
// TimeMarcher call sequence (TimeMarcher.F90:28-133) issued as sm_100a kernels on one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "afid_gpu.h"
#include "afid_internal.h"
#include "afid_salinity.h"

using namespace afid;


namespace {

int fail_cuda(afid_ctx_t *ctx, cudaError_t e) {
  if (ctx) ctx->last_cuda = e;
  return AFID_E_CUDA;
}

#define AFID_CUDA(ctx, call)                       \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return fail_cuda(ctx, e_); \
  } while (0)

bool make_plan(int n, FftPlan *p) {
  p->n = n;
  p->npass = 0;
  int m = n;
  while (m % 4 == 0 && p->npass < kMaxFftPasses) { p->radix[p->npass++] = 4; m /= 4; }
  while (m % 2 == 0 && p->npass < kMaxFftPasses) { p->radix[p->npass++] = 2; m /= 2; }
  while (m % 3 == 0 && p->npass < kMaxFftPasses) { p->radix[p->npass++] = 3; m /= 3; }
  while (m % 5 == 0 && p->npass < kMaxFftPasses) { p->radix[p->npass++] = 5; m /= 5; }
  return m == 1;
}

// exp(-2 pi i m / n) for m = 0..n-1
template <typename C>
std::vector<C> twiddles(int n) {
  std::vector<C> t(n);
  const double two_pi = 2.0 * 3.14159265358979323846264338327950288;
  for (int m = 0; m < n; ++m) {
    const double a = two_pi * (double)m / (double)n;
    t[m].x = (decltype(t[m].x))std::cos(a);
    t[m].y = (decltype(t[m].y))(-std::sin(a));
  }
  return t;
}

int round_up(int a, int b) { return (a + b - 1) / b * b; }

// Spacings and physics scalars of the geometry (everything but the sizes).
void geom_physics(Geom &g, const afid_grid_t *grid, const afid_params_t *prm) {
  g.dx = (double)g.nxm / grid->alx3;  // CreateGrid.F90:100-106
  g.dy = (double)g.nym / grid->ylen;
  g.dz = (double)g.nzm / grid->zlen;
  g.dyq = g.dy * g.dy;
  g.dzq = g.dz * g.dz;
  g.ren = prm->ren;
  g.pect = prm->pect;
  g.byct = prm->byct;
  g.rren = 1.0 / prm->ren;
  g.rpect = 1.0 / prm->pect;
  g.udyq_re = g.dyq / prm->ren;  // ExplicitTermsVX.F90:27-28
  g.udzq_re = g.dzq / prm->ren;
  g.udyq_pe = g.dyq / prm->pect;  // ExplicitTermsTemp.F90:24-25
  g.udzq_pe = g.dzq / prm->pect;
  // ExplicitTermsVY.F90:30-34
  g.gy = (prm->inslwn == 0 || prm->inslws == 0) ? prm->dpdy * prm->dpdy / (prm->ren * prm->ren)
                                                 : 8.0 * (prm->dpdy * prm->dpdy) / (prm->ren * prm->ren);
  g.xplusu = prm->xplusu;
  g.xminusu = prm->xminusu;
  g.active_t = prm->active_t;
  g.gaxis = prm->gaxis;
  g.inslws = prm->inslws;
  g.inslwn = prm->inslwn;
  g.tfixs = prm->tfixs;
  g.tfixn = prm->tfixn;
}

template <typename T>
cudaError_t dalloc(afid_ctx_t *ctx, T **p, size_t count) {
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) return e;
  ctx->allocs.push_back(q);
  ctx->dev_bytes += (long long)(std::max<size_t>(count, 1) * sizeof(T));
  *p = static_cast<T *>(q);
  return cudaMemset(q, 0, std::max<size_t>(count, 1) * sizeof(T));
}

// Copy a Fortran-layout host field (pointer at (1,1,1), leading dims ld_x, ld_y) into the
// device layout (ldx, nym); nx doubles per x-column.
int copy_field(afid_ctx_t *ctx, double *dst, const double *src, int ld_x, int ld_y, bool to_dev,
               double *hdst = nullptr) {
  const Geom &g = ctx->L.g;
  const size_t w = (size_t)g.nx * sizeof(double);
  cudaMemcpyKind kind = to_dev ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  if (ld_x == g.nx && ld_y == g.nym && g.nx != g.ldx && !g.batch) {
    // packed host array: one linear transfer through an intermediate buffer (free between
    // steps), repacked on the device; pitched copies of 2 KB rows run far below the link rate
    const size_t rows = (size_t)g.nym * g.nzm, bytes = rows * w;
    double *stage = ctx->vx_o;
    if (to_dev) {
      AFID_CUDA(ctx, cudaMemcpyAsync(stage, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
      AFID_CUDA(ctx, launch_repack(ctx->stream, stage, g.nx, dst, g.ldx, g.nx, rows));
    } else {
      AFID_CUDA(ctx, launch_repack(ctx->stream, dst, g.ldx, stage, g.nx, g.nx, rows));
      AFID_CUDA(ctx, cudaMemcpyAsync(hdst, stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    }
    ctx->launches += 1;
    return AFID_OK;
  }
  if (ld_y == g.nym) {
    if (to_dev)
      AFID_CUDA(ctx, cudaMemcpy2DAsync(dst, (size_t)g.ldx * sizeof(double), src, (size_t)ld_x * sizeof(double),
                                       w, (size_t)g.nym * g.nzm, kind, ctx->stream));
    else
      AFID_CUDA(ctx, cudaMemcpy2DAsync(hdst, (size_t)ld_x * sizeof(double), dst, (size_t)g.ldx * sizeof(double),
                                       w, (size_t)g.nym * g.nzm, kind, ctx->stream));
    return AFID_OK;
  }
  for (int i = 0; i < g.nzm; ++i) {
    const size_t hoff = (size_t)i * ld_x * ld_y;
    const size_t doff = (size_t)i * g.ldx * g.nym;
    if (to_dev)
      AFID_CUDA(ctx, cudaMemcpy2DAsync(dst + doff, (size_t)g.ldx * sizeof(double), src + hoff,
                                       (size_t)ld_x * sizeof(double), w, g.nym, kind, ctx->stream));
    else
      AFID_CUDA(ctx, cudaMemcpy2DAsync(hdst + hoff, (size_t)ld_x * sizeof(double), dst + doff,
                                       (size_t)g.ldx * sizeof(double), w, g.nym, kind, ctx->stream));
  }
  return AFID_OK;
}

int check_err_flag(afid_ctx_t *ctx) {
  int h = 0;
  AFID_CUDA(ctx, cudaMemcpyAsync(&h, ctx->err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  AFID_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h & 1) return AFID_E_SINGULAR;
  if (h & 2) return AFID_E_TIMEOUT;
  return AFID_OK;
}

SubstepBuffers buffers(afid_ctx_t *ctx) {
  SubstepBuffers b;
  b.sc = ctx->sc;
  b.cn_tab = ctx->cn_tab;
  b.vx = ctx->vx;
  b.vy = ctx->vy;
  b.vz = ctx->vz;
  b.temp = ctx->temp;
  b.pr = ctx->pr;
  b.rux = ctx->rux;
  b.ruy = ctx->ruy;
  b.ruz = ctx->ruz;
  b.rut = ctx->rut;
  b.vx_o = ctx->vx_o;
  b.vy_o = ctx->vy_o;
  b.vz_o = ctx->vz_o;
  b.temp_o = ctx->temp_o;
  b.spec = ctx->spec;
  b.phi = ctx->phi;
  b.err = ctx->err;
  return b;
}

cudaEvent_t next_event(afid_ctx_t *ctx, size_t *idx) {
  if (ctx->ev_used == ctx->ev_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    ctx->ev_pool.push_back(e);
  }
  *idx = ctx->ev_used;
  return ctx->ev_pool[ctx->ev_used++];
}

// Launch fn() and, when profiling, bracket it with events on the context stream.
template <typename F>
cudaError_t timed(afid_ctx_t *ctx, int cls, F fn) {
  if (!ctx->prof) return fn();
  size_t ia = 0, ib = 0;
  cudaEvent_t a = next_event(ctx, &ia);
  if (a) cudaEventRecord(a, ctx->stream);
  cudaError_t e = fn();
  cudaEvent_t b = next_event(ctx, &ib);
  if (b) cudaEventRecord(b, ctx->stream);
  if (a && b) ctx->recs.push_back({cls, ia, ib});
  return e;
}

int build_cn(afid_ctx_t *ctx, int ns0, int nsub, const double *al, const double *ga, const double *ro,
             double dt, double beta) {
  const Geom &g = ctx->L.g;
  CnInputs in;
  for (int m = 0; m < 3; ++m) {
    in.am[m] = ctx->am[m];
    in.ac[m] = ctx->ac[m];
    in.ap[m] = ctx->ap[m];
  }
  in.off[0] = 1;
  in.n[0] = g.nxm - 1;
  in.off[1] = 0;
  in.n[1] = g.nxm;
  in.off[2] = 0;
  in.n[2] = g.nxm;
  for (int s = 0; s < 3; ++s) {
    in.al[s] = s < nsub ? al[s] : 0.0;
    in.ga[s] = s < nsub ? ga[s] : 0.0;
    in.ro[s] = s < nsub ? ro[s] : 0.0;
  }
  in.dt = dt;
  in.beta = beta;
  in.pect = g.pect;
  in.ren = g.ren;
  in.ns0 = ns0;
  in.nsub = nsub;
  in.M = ctx->L.M;
  in.tab = ctx->cn_tab;
  in.sc = ctx->sc;
  AFID_CUDA(ctx, timed(ctx, 0, [&] { return launch_cn_tables(ctx->L, in); }));
  ctx->launches += 1;
  if (ctx->sal) {
    // SolveImpEqnUpdate_Sal (salinity.F90:408-425): one temperature-like matrix on the refined
    // rows with betadx = 0.5 al dt / pecs; its StepCoef carries alpec = al / pecs
    const SalCtx &S = *ctx->sal;
    CnInputs si = in;
    si.nmat = 1;
    si.am[0] = S.am_d;
    si.ac[0] = S.ac_d;
    si.ap[0] = S.ap_d;
    si.off[0] = 0;
    si.n[0] = S.sg.nxmr;
    si.pect = S.sg.pecs;
    si.M = S.sg.MR;
    si.tab = S.cn_tab;
    si.sc = S.sc;
    AFID_CUDA(ctx, timed(ctx, 0, [&] { return launch_cn_tables(ctx->L, si); }));
    ctx->launches += 1;
  }
  return AFID_OK;
}

// InterpVelMgrd + InterpSalMultigrid (TimeMarcher.F90:138-144) from the resident state.
int sal_interp(afid_ctx_t *ctx) {
  AFID_CUDA(ctx, timed(ctx, 10, [&] { return launch_sal_interp(ctx->L, *ctx->sal, ctx->vx, ctx->vy, ctx->vz); }));
  ctx->launches += kSalLaunchesInterp;
  return AFID_OK;
}

int run_substep(afid_ctx_t *ctx, int ns) {
  SubstepBuffers b = buffers(ctx);
  if (ctx->sal) {
    // ExplicitSalinity + ImplicitSalinity read the refined velocities and salc of the previous
    // substep only, so the salinity update goes first (TimeMarcher.F90:50-51, 95)
    AFID_CUDA(ctx, timed(ctx, 9, [&] { return launch_sal_step(ctx->L, *ctx->sal, ns); }));
    ctx->launches += 1;
  }
  for (int st = 0; st < kNumStages; ++st) {
    const Stage stage = static_cast<Stage>(st);
    if ((ctx->L.g.nzm == 1 || ctx->L.g.batch) && (stage == Stage::FftZFwd || stage == Stage::FftZInv)) continue;
    AFID_CUDA(ctx, timed(ctx, 1 + st, [&] { return launch_stage(ctx->L, b, ns, stage); }));
    ctx->launches += 1;
  }
  std::swap(ctx->temp, ctx->temp_o);  // temperature is final after K1; the state moves buffers
  if (ctx->sal) {
    std::swap(ctx->sal->sal, ctx->sal->sal_o);
    return sal_interp(ctx);
  }
  return AFID_OK;
}

void rk3(int nsst, double gam[3], double rom[3], double alm[3]) {
  // InitTimeMarchScheme.F90:16-49
  if (nsst > 1) {
    gam[0] = 8.0 / 15.0; gam[1] = 5.0 / 12.0; gam[2] = 3.0 / 4.0;
    rom[0] = 0.0; rom[1] = -17.0 / 60.0; rom[2] = -5.0 / 12.0;
  } else {
    gam[0] = 1.5; gam[1] = 0.0; gam[2] = 0.0;
    rom[0] = -0.5; rom[1] = 0.0; rom[2] = 0.0;
  }
  for (int n = 0; n < 3; ++n) alm[n] = gam[n] + rom[n];
}

}  // namespace

extern "C" {

const char *afid_gpu_status_string(int s) {
  switch (s) {
    case AFID_OK: return "ok";
    case AFID_E_ALLOC: return "allocation failure";
    case AFID_E_CFL: return "CFL number exceeds CFLMAX with fixed time step";
    case AFID_E_DTMIN: return "time step below DTMIN";
    case AFID_E_DIVERGENCE: return "maximum divergence exceeds RESID";
    case AFID_E_FFTSIZE: return "FFT size has a prime factor other than 2, 3, 5";
    case AFID_E_SINGULAR: return "singular Poisson mode (zero pivot)";
    case AFID_E_TIMEOUT: return "bounded device wait timed out";
    case AFID_E_INVALID: return "invalid argument or unsupported configuration";
    case AFID_E_CUDA: return "CUDA runtime error";
    case AFID_E_CAPACITY: return "capacity exhausted";
    case AFID_E_IO: return "restart file missing, unreadable or unsupported";
    case AFID_E_CANCELLED: return "job cancelled";
  }
  return "unknown status";
}

int afid_gpu_create(const afid_grid_t *grid, const afid_params_t *prm, afid_ctx_t **out) {
  return ctx_create(grid, prm, nullptr, out);
}

}  // extern "C"

namespace afid {

int ctx_create(const afid_grid_t *grid, const afid_params_t *prm, const BatchSpec *bs, afid_ctx_t **out) {
  if (!grid || !prm || !out) return AFID_E_INVALID;
  *out = nullptr;
  const int nxm = grid->nxm, nym = grid->nym, nzm = grid->nzm;
  if (nxm < 2 || nym < 1 || nzm < 1) return AFID_E_INVALID;
  if (prm->dpdz != 0.0) return AFID_E_INVALID;  // bulk-flux forcing (CorrectVelocity.F90:29-59) not on this path
  if (prm->gaxis == 2 && prm->inslwn == 1) return AFID_E_INVALID;  // mean-flux removal branch (CorrectVelocity.F90:62)
  if (prm->precision != AFID_PREC_FP64 && prm->precision != AFID_PREC_MIXED) return AFID_E_INVALID;
  const int M = cn_choose_M(nxm);
  if (M < 0) return AFID_E_INVALID;
  if (bs && (bs->ninst != nzm || !bs->inst || !bs->ak2)) return AFID_E_INVALID;
  FftPlan py, pz;
  if (!make_plan(nym, &py)) return AFID_E_FFTSIZE;
  if (bs) {
    pz.n = 1;  // instances do not couple along z: no z transform
    pz.npass = 0;
  } else if (!make_plan(nzm, &pz)) {
    return AFID_E_FFTSIZE;
  }

  afid_ctx_t *ctx = new (std::nothrow) afid_ctx_t();
  if (!ctx) return AFID_E_ALLOC;
  cudaGetDevice(&ctx->dev);
  ctx->nsst = prm->nsst > 1 ? 3 : 1;
  ctx->alx3 = grid->alx3;
  const bool mixed = prm->precision == AFID_PREC_MIXED;

  Geom g{};
  g.nxm = nxm;
  g.nym = nym;
  g.nzm = nzm;
  g.nx = nxm + 1;
  g.ldx = round_up(g.nx, 8);
  g.nyh = nym / 2 + 1;
  g.ldxc = round_up(nxm, 4);
  geom_physics(g, grid, prm);

  // One wall-normal column set must fit the shared memory of one block (3-D FP64: nxm <= ~850).
  int smem_optin = 0;
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->dev);
  if (smem_optin > 0 && k1_smem_bytes(g.ldx, M, mixed, bs != nullptr || nzm == 1) + 64 > (size_t)smem_optin) {
    afid_gpu_destroy(ctx);
    return AFID_E_INVALID;
  }
  const size_t nf = (size_t)g.ldx * nym * nzm;
  ctx->field_elems = nf;
  const size_t nspec = (size_t)g.ldxc * g.nyh * nzm;
  const size_t tsz = mixed ? sizeof(float) : sizeof(double);
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  chk(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
  ctx->stream = ctx->own_stream;
  chk(dalloc(ctx, &ctx->vx, nf));
  chk(dalloc(ctx, &ctx->vy, nf));
  chk(dalloc(ctx, &ctx->vz, nf));
  chk(dalloc(ctx, &ctx->temp, nf));
  chk(dalloc(ctx, &ctx->pr, nf));
  chk(dalloc(ctx, &ctx->vx_o, nf));
  chk(dalloc(ctx, &ctx->vy_o, nf));
  chk(dalloc(ctx, &ctx->vz_o, nf));
  chk(dalloc(ctx, &ctx->temp_o, nf));
  unsigned char *ru = nullptr;
  chk(dalloc(ctx, &ru, 4 * nf * tsz));
  ctx->rux = ru;
  ctx->ruy = ru + nf * tsz;
  ctx->ruz = ru + 2 * nf * tsz;
  ctx->rut = ru + 3 * nf * tsz;
  unsigned char *ph = nullptr;
  chk(dalloc(ctx, &ph, nf * tsz));
  ctx->phi = ph;
  unsigned char *sp = nullptr;
  chk(dalloc(ctx, &sp, nspec * 2 * tsz));
  ctx->spec = sp;
  const size_t nsets = bs ? (size_t)bs->ninst : 1;  // batch mode: one table set per instance
  chk(dalloc(ctx, &ctx->cn_tab, cn_tab_doubles(M, 3) * nsets));
  chk(dalloc(ctx, &ctx->sc, 3 * nsets));
  chk(dalloc(ctx, &ctx->err, 1));
  chk(dalloc(ctx, &ctx->red, 1));
  const int nb = globals_partial_blocks(g);
  chk(dalloc(ctx, &ctx->partial, (size_t)nb * 3));
  chk(dalloc(ctx, &ctx->gsum, 3));
  if (e == cudaSuccess) e = cudaMallocHost(&ctx->host_scratch, 8 * sizeof(double));

  // 1-D tables in one device block
  const int nx = g.nx;
  std::vector<double> h;
  auto put = [&](const double *src, int n, int len) -> size_t {
    while (h.size() % 8) h.push_back(0.0);  // 64-byte aligned tables (vector loads)
    size_t off = h.size();
    for (int k = 0; k < len; ++k) h.push_back((src && k < n) ? src[k] : 0.0);
    return off;
  };
  const int L1 = nx + 8;
  size_t o_udx3c = put(grid->udx3c, nx, L1), o_udx3m = put(grid->udx3m, nxm, L1);
  std::vector<double> idx(nxm);
  for (int k = 0; k < nxm; ++k) idx[k] = 1.0 / grid->udx3m[k];  // ExplicitTermsVX.F90:30-32
  size_t o_idx = put(idx.data(), nxm, L1);
  size_t o_ap3ck = put(grid->ap3ck, nx, L1), o_ac3ck = put(grid->ac3ck, nx, L1), o_am3ck = put(grid->am3ck, nx, L1);
  size_t o_ap3sk = put(grid->ap3sk, nxm, L1), o_ac3sk = put(grid->ac3sk, nxm, L1), o_am3sk = put(grid->am3sk, nxm, L1);
  size_t o_ap3ssk = put(grid->ap3ssk, nxm, L1), o_ac3ssk = put(grid->ac3ssk, nxm, L1),
         o_am3ssk = put(grid->am3ssk, nxm, L1);
  size_t o_amphk = put(grid->amphk, nxm, L1), o_acphk = put(grid->acphk, nxm, L1), o_apphk = put(grid->apphk, nxm, L1);
  size_t o_ak1 = bs ? put(nullptr, 0, nzm) : put(grid->ak1, nzm, nzm);
  size_t o_ak2 = bs ? put(bs->ak2, nym * nzm, nym * nzm) : put(grid->ak2, nym, nym);
  size_t o_g3rc = put(grid->g3rc, nx, L1);
  // g3rm from the cell centres as CreateGrid.F90 builds it (xm[nx-1] is the ghost centre)
  std::vector<double> g3rm(nx, 0.0);
  if (grid->xm && grid->xc) {
    for (int kc = 1; kc < nxm; ++kc) g3rm[kc] = (grid->xm[kc + 1] - grid->xm[kc - 1]) * g.dx * 0.5;
    g3rm[0] = (grid->xm[1] - (2 * grid->xc[0] - grid->xm[0])) * g.dx * 0.5;
  }
  size_t o_g3rm = put(g3rm.data(), nx, L1);
  std::vector<double> tbp((size_t)nym * nzm, 0.5), ttp((size_t)nym * nzm, -0.5);
  const double *src_bp = bs ? bs->tempbp : prm->tempbp, *src_tp = bs ? bs->temptp : prm->temptp;
  if (src_bp) std::memcpy(tbp.data(), src_bp, tbp.size() * sizeof(double));
  if (src_tp) std::memcpy(ttp.data(), src_tp, ttp.size() * sizeof(double));
  size_t o_tbp = put(tbp.data(), (int)tbp.size(), (int)tbp.size());
  size_t o_ttp = put(ttp.data(), (int)ttp.size(), (int)ttp.size());
  double *dtab = nullptr;
  if (e == cudaSuccess) e = dalloc(ctx, &dtab, h.size());
  if (e == cudaSuccess) e = cudaMemcpy(dtab, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
  Tables t{};
  if (dtab) {
    t.udx3c = dtab + o_udx3c;
    t.udx3m = dtab + o_udx3m;
    t.idx = dtab + o_idx;
    t.ap3ck = dtab + o_ap3ck;
    t.ac3ck = dtab + o_ac3ck;
    t.am3ck = dtab + o_am3ck;
    t.ap3sk = dtab + o_ap3sk;
    t.ac3sk = dtab + o_ac3sk;
    t.am3sk = dtab + o_am3sk;
    t.ap3ssk = dtab + o_ap3ssk;
    t.ac3ssk = dtab + o_ac3ssk;
    t.am3ssk = dtab + o_am3ssk;
    t.amphk = dtab + o_amphk;
    t.acphk = dtab + o_acphk;
    t.apphk = dtab + o_apphk;
    t.ak1 = dtab + o_ak1;
    t.ak2 = dtab + o_ak2;
    t.g3rc = dtab + o_g3rc;
    t.g3rm = dtab + o_g3rm;
    t.tempbp = dtab + o_tbp;
    t.temptp = dtab + o_ttp;
    ctx->am[0] = t.am3ck; ctx->ac[0] = t.ac3ck; ctx->ap[0] = t.ap3ck;
    ctx->am[1] = t.am3sk; ctx->ac[1] = t.ac3sk; ctx->ap[1] = t.ap3sk;
    ctx->am[2] = t.am3ssk; ctx->ac[2] = t.ac3ssk; ctx->ap[2] = t.ap3ssk;
  }
  // twiddles
  void *twy = nullptr, *twz = nullptr;
  if (e == cudaSuccess) {
    if (mixed) {
      auto a = twiddles<float2>(nym), b = twiddles<float2>(nzm);
      float2 *dy_ = nullptr, *dz_ = nullptr;
      e = dalloc(ctx, &dy_, a.size());
      if (e == cudaSuccess) e = dalloc(ctx, &dz_, b.size());
      if (e == cudaSuccess) e = cudaMemcpy(dy_, a.data(), a.size() * sizeof(float2), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = cudaMemcpy(dz_, b.data(), b.size() * sizeof(float2), cudaMemcpyHostToDevice);
      twy = dy_;
      twz = dz_;
    } else {
      auto a = twiddles<double2>(nym), b = twiddles<double2>(nzm);
      double2 *dy_ = nullptr, *dz_ = nullptr;
      e = dalloc(ctx, &dy_, a.size());
      if (e == cudaSuccess) e = dalloc(ctx, &dz_, b.size());
      if (e == cudaSuccess) e = cudaMemcpy(dy_, a.data(), a.size() * sizeof(double2), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = cudaMemcpy(dz_, b.data(), b.size() * sizeof(double2), cudaMemcpyHostToDevice);
      twy = dy_;
      twz = dz_;
    }
  }
  if (e != cudaSuccess) {
    ctx->last_cuda = e;
    afid_gpu_destroy(ctx);
    return (e == cudaErrorMemoryAllocation) ? AFID_E_ALLOC : AFID_E_CUDA;
  }
  LaunchCtx &L = ctx->L;
  L.g = g;
  L.t = t;
  L.stream = ctx->stream;
  L.M = M;
  L.mixed = mixed;
  const size_t csz = mixed ? sizeof(float2) : sizeof(double2);
  const size_t smem_cap = 96 * 1024;
  L.tx_y = 8;
  while (L.tx_y > 2 && (size_t)L.tx_y * nym * csz > smem_cap) L.tx_y /= 2;
  L.tx_z = 8;
  while (L.tx_z > 2 && (size_t)2 * L.tx_z * nzm * csz > smem_cap) L.tx_z /= 2;
  if ((size_t)L.tx_y * nym * csz > 200 * 1024 || (!bs && (size_t)2 * L.tx_z * nzm * csz > 200 * 1024)) {
    afid_gpu_destroy(ctx);
    return AFID_E_INVALID;
  }
  if (bs) {
    ctx->ninst = bs->ninst;
    cudaError_t eb = dalloc(ctx, &ctx->inst_dev, (size_t)bs->ninst);
    if (eb == cudaSuccess)
      eb = cudaMemcpy(ctx->inst_dev, bs->inst, sizeof(InstScal) * bs->ninst, cudaMemcpyHostToDevice);
    if (eb == cudaSuccess) eb = dalloc(ctx, &ctx->active_dev, (size_t)bs->ninst);
    if (eb == cudaSuccess) eb = cudaMemset(ctx->active_dev, 1, bs->ninst);
    if (eb != cudaSuccess) {
      ctx->last_cuda = eb;
      afid_gpu_destroy(ctx);
      return eb == cudaErrorMemoryAllocation ? AFID_E_ALLOC : AFID_E_CUDA;
    }
    L.g.batch = 1;
    L.g.inst = ctx->inst_dev;
    L.g.active = ctx->active_dev;
  }
  L.warp_fft = true;
  L.k1_var = 0;
  L.k4_var = 0;
  L.fftz_var = 0;
  L.ify_var = 0;
  L.div_var = 0;
  L.plan_y = py;
  L.plan_z = pz;
  L.twy = twy;
  L.twz = twz;
  *out = ctx;
  return AFID_OK;
}

SubstepBuffers ctx_buffers(afid_ctx_t *ctx) { return buffers(ctx); }
int ctx_run_substep(afid_ctx_t *ctx, int ns) { return run_substep(ctx, ns); }
int ctx_fail(afid_ctx_t *ctx, cudaError_t e) { return fail_cuda(ctx, e); }

// Time every K1 thread shape on the first `sample` columns and keep the fastest.  The RK3
// histories point at scratch memory for these launches (K1 updates them in place); the other
// outputs are intermediates of the next substep or the idle temperature buffer, which the next
// K1 overwrites, so the state is untouched.  Idle batch slots are timed as active.
int ctx_autotune(afid_ctx_t *ctx, bool force) {
  if (ctx->tuned && !force) return AFID_OK;
  LaunchCtx L = ctx->L;
  int tpc[AFID_TUNE_MAX] = {0}, rpt[AFID_TUNE_MAX] = {0}, cap[AFID_TUNE_MAX] = {0}, pol[AFID_TUNE_MAX] = {0};
  const int n = k1_shapes(L.M, tpc, rpt, cap, pol);
  afid_tune_info_t info{};
  info.ncand = n;
  const int ncol = L.g.nym * L.g.nzm;
  const int sample = std::min(ncol, 148 * 24);
  info.sample_columns = sample;
  for (int v = 0; v < AFID_TUNE_MAX; ++v) {
    info.threads[v] = v < n ? tpc[v] : 0;
    info.rows[v] = v < n ? rpt[v] : 0;
    info.regcap[v] = v < n ? cap[v] : 0;
    info.policy[v] = v < n ? pol[v] : 0;
    info.us[v] = -1.0;
  }
  if (n > 1) {
    const size_t tsz = L.mixed ? sizeof(float) : sizeof(double);
    const size_t per = (size_t)sample * L.g.ldx * tsz;
    char *scratch = nullptr;
    AFID_CUDA(ctx, cudaMalloc(&scratch, 4 * per));
    SubstepBuffers b = buffers(ctx);
    b.rux = scratch;
    b.ruy = scratch + per;
    b.ruz = scratch + 2 * per;
    b.rut = scratch + 3 * per;
    L.g.active = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMemsetAsync(scratch, 0, 4 * per, ctx->stream);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    double best = 1e300;
    constexpr int kReps = 5;
    // two rounds over all candidates, keeping each one's best: the first round also brings the
    // clocks up, which would otherwise bias against the first candidates
    for (int round = 0; round < 2 && e == cudaSuccess; ++round) {
      for (int v = 0; v < n && e == cudaSuccess; ++v) {
        auto run = [&] { return L.mixed ? launch_k1_mixed(L, b, 0, v, sample) : launch_k1_fp64(L, b, 0, v, sample); };
        if (!k1_shape_usable(L.M, v, L.g.batch != 0, L.g.nzm == 1 || L.g.batch)) continue;
        if (run() != cudaSuccess) {  // this shape does not fit the device: skip it
          cudaGetLastError();
          continue;
        }
        ctx->launches += 1 + kReps;
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < kReps; ++r) run();
        cudaEventRecord(e1, ctx->stream);
        e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) break;
        const double us = 1e3 * ms / kReps;
        if (info.us[v] < 0.0 || us < info.us[v]) info.us[v] = us;
      }
    }
    for (int v = 0; v < n; ++v)
      if (info.us[v] >= 0.0 && info.us[v] < best) {
        best = info.us[v];
        info.chosen = v;
      }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaError_t ef = cudaFree(scratch);
    if (e == cudaSuccess) e = ef;
    if (e != cudaSuccess) return fail_cuda(ctx, e);
  }
  ctx->L.k1_var = info.chosen;
  // The Poisson tridiagonal: both forms timed on full launches over the spectrum buffer, whose
  // contents are dead between substeps (K2 rewrites all of it).
  info.k4_chosen = 0;
  info.k4_us[0] = info.k4_us[1] = -1.0;
  {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    SubstepBuffers b = buffers(ctx);
    LaunchCtx L4 = ctx->L;
    L4.g.active = ctx->L.g.active;
    constexpr int kReps = 3;
    for (int round = 0; round < 2 && e == cudaSuccess; ++round)
      for (int v = 0; v < 2 && e == cudaSuccess; ++v) {
        L4.k4_var = v;
        if (launch_stage(L4, b, 0, Stage::Tridiag) != cudaSuccess) {  // this form does not fit: skip it
          cudaGetLastError();
          continue;
        }
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < kReps && e == cudaSuccess; ++r) e = launch_stage(L4, b, 0, Stage::Tridiag);
        cudaEventRecord(e1, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        ctx->launches += 1 + kReps;
        const double us = 1e3 * ms / kReps;
        if (e == cudaSuccess && (info.k4_us[v] < 0.0 || us < info.k4_us[v])) info.k4_us[v] = us;
      }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    if (info.k4_us[1] >= 0.0 && info.k4_us[1] < info.k4_us[0]) info.k4_chosen = 1;
  }
  ctx->L.k4_var = info.k4_chosen;
  // The z transforms (3-D single domains): one tile per block, or persistent blocks with the next
  // tile's copies in flight; timed the same way (the spectrum's contents are dead here too).
  info.fftz_chosen = 0;
  info.fftz_us[0] = info.fftz_us[1] = info.fftz_us[2] = -1.0;
  if (ctx->L.g.nzm > 1 && !ctx->L.g.batch) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    SubstepBuffers b = buffers(ctx);
    LaunchCtx Lz = ctx->L;
    constexpr int kReps = 3;
    for (int round = 0; round < 2 && e == cudaSuccess; ++round)
      for (int v = 0; v < 3 && e == cudaSuccess; ++v) {
        Lz.fftz_var = v;
        if (launch_stage(Lz, b, 0, Stage::FftZFwd) != cudaSuccess) {  // this form does not fit: skip it
          cudaGetLastError();
          continue;
        }
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < kReps && e == cudaSuccess; ++r) e = launch_stage(Lz, b, 0, Stage::FftZFwd);
        cudaEventRecord(e1, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        ctx->launches += 1 + kReps;
        const double us = 1e3 * ms / kReps;
        if (e == cudaSuccess && (info.fftz_us[v] < 0.0 || us < info.fftz_us[v])) info.fftz_us[v] = us;
      }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    for (int v = 1; v < 3; ++v)
      if (info.fftz_us[v] >= 0.0 && info.fftz_us[v] < info.fftz_us[info.fftz_chosen]) info.fftz_chosen = v;
  }
  ctx->L.fftz_var = info.fftz_chosen;
  // The inverse y transform (FP64 single domains): per-thread copies or tensor copies, timed on
  // full launches (phi and the spectrum are dead here: K6 rewrites phi from the spectrum).
  info.ify_chosen = 0;
  info.ify_us[0] = info.ify_us[1] = -1.0;
  if (!ctx->L.mixed && !ctx->L.g.batch && ctx->L.warp_fft) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    SubstepBuffers b = buffers(ctx);
    LaunchCtx L6 = ctx->L;
    constexpr int kReps = 3;
    for (int round = 0; round < 2 && e == cudaSuccess; ++round)
      for (int v = 0; v < 2 && e == cudaSuccess; ++v) {
        L6.ify_var = v;
        if (launch_stage(L6, b, 0, Stage::IfftY) != cudaSuccess) {  // this form does not apply: skip it
          cudaGetLastError();
          continue;
        }
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < kReps && e == cudaSuccess; ++r) e = launch_stage(L6, b, 0, Stage::IfftY);
        cudaEventRecord(e1, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        ctx->launches += 1 + kReps;
        const double us = 1e3 * ms / kReps;
        if (e == cudaSuccess && (info.ify_us[v] < 0.0 || us < info.ify_us[v])) info.ify_us[v] = us;
      }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    if (info.ify_us[1] >= 0.0 && info.ify_us[1] < info.ify_us[0]) info.ify_chosen = 1;
  }
  ctx->L.ify_var = info.ify_chosen;
  // The divergence + forward y transform (FP64 single domains): per-thread loads or tensor
  // copies, timed on full launches (the spectrum is dead here: K2 rewrites it).
  info.div_chosen = 0;
  info.div_us[0] = info.div_us[1] = -1.0;
  if (!ctx->L.mixed && !ctx->L.g.batch && ctx->L.warp_fft) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    SubstepBuffers b = buffers(ctx);
    LaunchCtx L2 = ctx->L;
    constexpr int kReps = 3;
    for (int round = 0; round < 2 && e == cudaSuccess; ++round)
      for (int v = 0; v < 2 && e == cudaSuccess; ++v) {
        L2.div_var = v;
        if (launch_stage(L2, b, 0, Stage::DivFftY) != cudaSuccess) {  // this form does not apply: skip it
          cudaGetLastError();
          continue;
        }
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < kReps && e == cudaSuccess; ++r) e = launch_stage(L2, b, 0, Stage::DivFftY);
        cudaEventRecord(e1, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        ctx->launches += 1 + kReps;
        const double us = 1e3 * ms / kReps;
        if (e == cudaSuccess && (info.div_us[v] < 0.0 || us < info.div_us[v])) info.div_us[v] = us;
      }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    if (info.div_us[1] >= 0.0 && info.div_us[1] < info.div_us[0]) info.div_chosen = 1;
  }
  ctx->L.div_var = info.div_chosen;
  ctx->tune = info;
  ctx->tuned = true;
  return check_err_flag(ctx);
}

// New physics for a single-domain context of the same grid (sizes and wall-normal tables
// unchanged): scalars, wavenumbers and plate temperatures.  Launches captured before this call
// keep the old scalars.
int ctx_update_params(afid_ctx_t *ctx, const afid_grid_t *grid, const afid_params_t *prm) {
  Geom &g = ctx->L.g;
  if (g.batch || grid->nxm != g.nxm || grid->nym != g.nym || grid->nzm != g.nzm || grid->alx3 != ctx->alx3)
    return AFID_E_INVALID;
  if (prm->dpdz != 0.0 || (prm->gaxis == 2 && prm->inslwn == 1)) return AFID_E_INVALID;
  const Tables &t = ctx->L.t;
  const size_t ny = (size_t)g.nym, nz = (size_t)g.nzm;
  std::vector<double> bp(ny * nz, 0.5), tp(ny * nz, -0.5);
  if (prm->tempbp) std::memcpy(bp.data(), prm->tempbp, bp.size() * sizeof(double));
  if (prm->temptp) std::memcpy(tp.data(), prm->temptp, tp.size() * sizeof(double));
  AFID_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  AFID_CUDA(ctx, cudaMemcpy(const_cast<double *>(t.ak1), grid->ak1, nz * sizeof(double), cudaMemcpyHostToDevice));
  AFID_CUDA(ctx, cudaMemcpy(const_cast<double *>(t.ak2), grid->ak2, ny * sizeof(double), cudaMemcpyHostToDevice));
  AFID_CUDA(ctx, cudaMemcpy(const_cast<double *>(t.tempbp), bp.data(), bp.size() * sizeof(double), cudaMemcpyHostToDevice));
  AFID_CUDA(ctx, cudaMemcpy(const_cast<double *>(t.temptp), tp.data(), tp.size() * sizeof(double), cudaMemcpyHostToDevice));
  geom_physics(g, grid, prm);
  return AFID_OK;
}

// CN tables and RK3 coefficients of all substeps for every instance of a batch, dt from the device.
int ctx_build_cn_batch(afid_ctx_t *ctx, const double *dt_dev) {
  const Geom &g = ctx->L.g;
  CnInputs in;
  for (int m = 0; m < 3; ++m) {
    in.am[m] = ctx->am[m];
    in.ac[m] = ctx->ac[m];
    in.ap[m] = ctx->ap[m];
  }
  in.off[0] = 1;
  in.n[0] = g.nxm - 1;
  in.off[1] = 0;
  in.n[1] = g.nxm;
  in.off[2] = 0;
  in.n[2] = g.nxm;
  double gam[3], rom[3], alm[3];
  rk3(ctx->nsst, gam, rom, alm);
  for (int s2 = 0; s2 < 3; ++s2) {
    in.al[s2] = alm[s2];
    in.ga[s2] = gam[s2];
    in.ro[s2] = rom[s2];
  }
  in.dt = 0.0;
  in.beta = 0.0;
  in.pect = g.pect;
  in.ren = g.ren;
  in.ns0 = 0;
  in.nsub = ctx->nsst;
  in.M = ctx->L.M;
  in.tab = ctx->cn_tab;
  in.sc = ctx->sc;
  in.dt_dev = dt_dev;
  in.inst = ctx->inst_dev;
  in.active = ctx->active_dev;
  in.ninst = ctx->ninst;
  AFID_CUDA(ctx, timed(ctx, 0, [&] { return launch_cn_tables(ctx->L, in); }));
  ctx->launches += 1;
  return AFID_OK;
}

}  // namespace afid

extern "C" {

int afid_gpu_destroy(afid_ctx_t *ctx) {
  if (!ctx) return AFID_OK;
  cudaSetDevice(ctx->dev);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (void *p : ctx->allocs) cudaFree(p);
  delete ctx->sal;
  if (ctx->stats_buf) cudaFree(ctx->stats_buf);
  if (ctx->spec_acc) cudaFree(ctx->spec_acc);
  for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
  if (ctx->host_scratch) cudaFreeHost(ctx->host_scratch);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return AFID_OK;
}

int afid_gpu_set_stream(afid_ctx_t *ctx, void *stream) {
  if (!ctx) return AFID_E_INVALID;
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  ctx->L.stream = ctx->stream;
  return AFID_OK;
}

void *afid_gpu_get_stream(afid_ctx_t *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int afid_gpu_set_wait_test(afid_ctx_t *ctx, long long polls) {
  if (!ctx || polls < 0 || polls > (1LL << 24)) return AFID_E_INVALID;
  ctx->L.g.wait_test_polls = polls;
  return AFID_OK;
}

int afid_gpu_synchronize(afid_ctx_t *ctx) {
  if (!ctx) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  return check_err_flag(ctx);
}

int afid_gpu_upload(afid_ctx_t *ctx, const double *vx, const double *vy, const double *vz,
                    const double *temp, const double *pr, int ld_x, int ld_y) {
  if (!ctx) return AFID_E_INVALID;
  const Geom &g = ctx->L.g;
  if (ld_x < g.nx || ld_y < g.nym) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  int s;
  if (vx && (s = copy_field(ctx, ctx->vx, vx, ld_x, ld_y, true)) != AFID_OK) return s;
  if (vy && (s = copy_field(ctx, ctx->vy, vy, ld_x, ld_y, true)) != AFID_OK) return s;
  if (vz && (s = copy_field(ctx, ctx->vz, vz, ld_x, ld_y, true)) != AFID_OK) return s;
  if (temp && (s = copy_field(ctx, ctx->temp, temp, ld_x, ld_y, true)) != AFID_OK) return s;
  if (pr && (s = copy_field(ctx, ctx->pr, pr, ld_x, ld_y, true)) != AFID_OK) return s;
  const size_t tsz = ctx->L.mixed ? sizeof(float) : sizeof(double);
  AFID_CUDA(ctx, cudaMemsetAsync(ctx->rux, 0, 4 * ctx->field_elems * tsz, ctx->stream));
  if (ctx->sal && (s = sal_interp(ctx)) != AFID_OK) return s;  // the refined velocities follow
  AFID_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return AFID_OK;
}

int afid_gpu_download(afid_ctx_t *ctx, double *vx, double *vy, double *vz, double *temp, double *pr,
                      int ld_x, int ld_y) {
  if (!ctx) return AFID_E_INVALID;
  const Geom &g = ctx->L.g;
  if (ld_x < g.nx || ld_y < g.nym) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  int s;
  if (vx && (s = copy_field(ctx, ctx->vx, nullptr, ld_x, ld_y, false, vx)) != AFID_OK) return s;
  if (vy && (s = copy_field(ctx, ctx->vy, nullptr, ld_x, ld_y, false, vy)) != AFID_OK) return s;
  if (vz && (s = copy_field(ctx, ctx->vz, nullptr, ld_x, ld_y, false, vz)) != AFID_OK) return s;
  if (temp && (s = copy_field(ctx, ctx->temp, nullptr, ld_x, ld_y, false, temp)) != AFID_OK) return s;
  if (pr && (s = copy_field(ctx, ctx->pr, nullptr, ld_x, ld_y, false, pr)) != AFID_OK) return s;
  return check_err_flag(ctx);
}

int afid_gpu_timemarcher(afid_ctx_t *ctx, double dt, int ntime) {
  (void)ntime;
  if (!ctx || !(dt > 0.0)) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  double gam[3], rom[3], alm[3];
  rk3(ctx->nsst, gam, rom, alm);
  const double beta = dt / ctx->L.g.ren * 0.5;  // TimeMarcher.F90:28
  int s;
  if ((s = build_cn(ctx, 0, ctx->nsst, alm, gam, rom, dt, beta)) != AFID_OK) return s;
  if ((s = ctx_autotune(ctx, false)) != AFID_OK) return s;
  for (int ns = 0; ns < ctx->nsst; ++ns)
    if ((s = run_substep(ctx, ns)) != AFID_OK) return s;
  return AFID_OK;
}

int afid_gpu_substep(afid_ctx_t *ctx, int ns, double al, double ga, double ro, double dt, double beta) {
  if (!ctx || ns < 0 || ns > 2 || !(dt > 0.0)) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  int s;
  if ((s = build_cn(ctx, ns, 1, &al, &ga, &ro, dt, beta)) != AFID_OK) return s;
  if ((s = ctx_autotune(ctx, false)) != AFID_OK) return s;
  return run_substep(ctx, ns);
}

int afid_gpu_cfl(afid_ctx_t *ctx, double *cflm) {
  if (!ctx || !cflm) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  AFID_CUDA(ctx, timed(ctx, 8, [&] { return launch_max_reduce(ctx->L, false, ctx->vx, ctx->vy, ctx->vz, ctx->red); }));
  ctx->launches += 1;
  AFID_CUDA(ctx, cudaMemcpyAsync(ctx->host_scratch, ctx->red, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  int s = check_err_flag(ctx);
  const double v = ctx->host_scratch[0];
  *cflm = (v != v) ? v : std::max(0.00000001, v);  // CalcMaxCFL.F90:22; a NaN maximum is passed on
  return s;
}

int afid_gpu_divmax(afid_ctx_t *ctx, double *dmax) {
  if (!ctx || !dmax) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  AFID_CUDA(ctx, timed(ctx, 8, [&] { return launch_max_reduce(ctx->L, true, ctx->vx, ctx->vy, ctx->vz, ctx->red); }));
  ctx->launches += 1;
  AFID_CUDA(ctx, cudaMemcpyAsync(ctx->host_scratch, ctx->red, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  int s = check_err_flag(ctx);
  *dmax = ctx->host_scratch[0];
  return s;
}

int afid_gpu_globals(afid_ctx_t *ctx, double ra_pr, double *nu_vol, double *ke, double *tmean) {
  if (!ctx) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  const Geom &g = ctx->L.g;
  AFID_CUDA(ctx, timed(ctx, 8, [&] {
    return launch_globals(ctx->L, ctx->vx, ctx->vy, ctx->vz, ctx->temp, ctx->partial, ctx->gsum);
  }));
  ctx->launches += 2;
  AFID_CUDA(ctx, cudaMemcpyAsync(ctx->host_scratch, ctx->gsum, 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
  int s = check_err_flag(ctx);
  // GlobalQuantities.F90:35,79,87-91
  const double vol = 1.0 / (ctx->alx3 * g.dx * (double)g.nzm * (double)g.nym);
  if (nu_vol) *nu_vol = 1.0 + std::sqrt(ra_pr) * ctx->host_scratch[0] * vol;
  if (ke) *ke = 0.5 * ctx->host_scratch[1] * vol;
  if (tmean) *tmean = ctx->host_scratch[2] * vol;
  return s;
}

int afid_gpu_cuda_error(afid_ctx_t *ctx) { return ctx ? (int)ctx->last_cuda : 0; }

int afid_gpu_dims(afid_ctx_t *ctx, int dims[6]) {
  if (!ctx || !dims) return AFID_E_INVALID;
  dims[0] = ctx->L.g.nxm;
  dims[1] = ctx->L.g.nym;
  dims[2] = ctx->L.g.nzm;
  dims[3] = ctx->sal ? ctx->sal->sg.nxmr : 0;
  dims[4] = ctx->sal ? ctx->sal->sg.nymr : 0;
  dims[5] = ctx->sal ? ctx->sal->sg.nzmr : 0;
  return AFID_OK;
}

int afid_gpu_field_device_ptr(afid_ctx_t *ctx, int which, void **dptr, int *ldx) {
  if (!ctx || !dptr) return AFID_E_INVALID;
  double *p = nullptr;
  switch (which) {
    case 0: p = ctx->vx; break;
    case 1: p = ctx->vy; break;
    case 2: p = ctx->vz; break;
    case 3: p = ctx->temp; break;
    case 4: p = ctx->pr; break;
    default: return AFID_E_INVALID;
  }
  *dptr = p;
  if (ldx) *ldx = ctx->L.g.ldx;
  return AFID_OK;
}

long long afid_gpu_launch_count(afid_ctx_t *ctx) { return ctx ? ctx->launches : 0; }

int afid_gpu_set_k1_shape(afid_ctx_t *ctx, int index) {
  if (!ctx) return AFID_E_INVALID;
  int tpc[AFID_TUNE_MAX], rpt[AFID_TUNE_MAX], cap[AFID_TUNE_MAX], pol[AFID_TUNE_MAX];
  const int n = k1_shapes(ctx->L.M, tpc, rpt, cap, pol);
  if (index < 0 || index >= n) return AFID_E_INVALID;
  const bool two_d = ctx->L.g.nzm == 1 || ctx->L.g.batch;
  if (!k1_shape_usable(ctx->L.M, index, ctx->L.g.batch != 0, two_d)) return AFID_E_INVALID;
  afid_tune_info_t info{};
  info.ncand = n;
  info.chosen = index;
  for (int v = 0; v < AFID_TUNE_MAX; ++v) {
    info.threads[v] = v < n ? tpc[v] : 0;
    info.rows[v] = v < n ? rpt[v] : 0;
    info.regcap[v] = v < n ? cap[v] : 0;
    info.policy[v] = v < n ? pol[v] : 0;
    info.us[v] = -1.0;
  }
  ctx->tune = info;
  ctx->L.k1_var = index;
  ctx->tuned = true;
  return AFID_OK;
}

int afid_gpu_set_k4_form(afid_ctx_t *ctx, int form) {
  if (!ctx || form < 0 || form > 1) return AFID_E_INVALID;
  ctx->L.k4_var = form;
  ctx->tune.k4_chosen = form;
  return AFID_OK;
}

int afid_gpu_set_fftz_form(afid_ctx_t *ctx, int form) {
  if (!ctx || form < 0 || form > 2) return AFID_E_INVALID;
  // the persistent forms hold two tiles of nzm rows in shared memory: 8 elements a row, or 128
  // bytes a row for the tensor-copy form, with its barriers and 1024-byte alignment slack
  const size_t elem = ctx->L.mixed ? 8 : 16;
  const size_t tiles = form == 2 ? 2 * (size_t)ctx->L.g.nzm * 128 + 16 + 1024 : 2 * (size_t)ctx->L.g.nzm * 8 * elem;
  if (form > 0 && tiles > (size_t)227 * 1024) return AFID_E_INVALID;
  ctx->L.fftz_var = form;
  ctx->tune.fftz_chosen = form;
  return AFID_OK;
}

int afid_gpu_set_ify_form(afid_ctx_t *ctx, int form) {
  if (!ctx || form < 0 || form > 1) return AFID_E_INVALID;
  // the tensor-copy form: FP64 single domains whose y transform is a warp FFT of at most 384
  // points (N = 32 x {1, 2, 3, 4, 6, 8, 12})
  const int nym = ctx->L.g.nym, n1 = nym / 32;
  const bool fits = nym % 32 == 0 && (n1 <= 4 || n1 == 6 || n1 == 8 || n1 == 12);
  if (form == 1 && (ctx->L.mixed || ctx->L.g.batch || !ctx->L.warp_fft || !fits)) return AFID_E_INVALID;
  ctx->L.ify_var = form;
  ctx->tune.ify_chosen = form;
  return AFID_OK;
}

int afid_gpu_set_div_form(afid_ctx_t *ctx, int form) {
  if (!ctx || form < 0 || form > 1) return AFID_E_INVALID;
  // the tensor-copy form: FP64 single domains whose y transform is a warp FFT (nym = 32 x N1)
  if (form == 1 && (ctx->L.mixed || ctx->L.g.batch || !ctx->L.warp_fft || ctx->L.g.nym % 32 != 0))
    return AFID_E_INVALID;
  ctx->L.div_var = form;
  ctx->tune.div_chosen = form;
  return AFID_OK;
}

int afid_gpu_autotune(afid_ctx_t *ctx, int force, afid_tune_info_t *info) {
  if (!ctx) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  const int s = ctx_autotune(ctx, force != 0);
  if (info) *info = ctx->tune;
  return s;
}

int afid_gpu_profile_enable(afid_ctx_t *ctx, int enable) {
  if (!ctx) return AFID_E_INVALID;
  ctx->prof = enable != 0;
  return AFID_OK;
}

int afid_gpu_profile_report(afid_ctx_t *ctx, double *ms, long long *count, int n) {
  if (!ctx) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  AFID_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int c = 0; c < n; ++c) {
    if (ms) ms[c] = 0.0;
    if (count) count[c] = 0;
  }
  for (const auto &r : ctx->recs) {
    if (r.cls >= n) continue;
    float t = 0.f;
    AFID_CUDA(ctx, cudaEventElapsedTime(&t, ctx->ev_pool[r.a], ctx->ev_pool[r.b]));
    if (ms) ms[r.cls] += t;
    if (count) count[r.cls] += 1;
  }
  ctx->recs.clear();
  ctx->ev_used = 0;
  return AFID_OK;
}

}  // extern "C"

// ==========================================================================================
// Multi-resolution salinity (include/afid_salinity.h)
// ==========================================================================================
namespace {

bool stencil_ok(const afid_stencil_t &s, int n, int lo, int hi) {
  if (s.n != n || !s.start || !s.w) return false;
  for (int t = 0; t < n; ++t)
    if (s.start[t] < lo || s.start[t] > hi) return false;
  return true;
}

// Refined field <-> Fortran-layout host array (rows x nymr x nzmr, leading dims ld_x, ld_y).
// A packed host array (ld_x == rows, ld_y == nymr) with a staging buffer travels as one linear
// copy plus an on-device repack, as the coarse fields do; otherwise one pitched copy per z-plane.
int sal_copy(afid_ctx_t *ctx, double *dev, int rows, const double *src, double *hdst, int ld_x, int ld_y,
             bool to_dev, double *stage = nullptr) {
  const SalGeom &sg = ctx->sal->sg;
  const size_t w = (size_t)rows * sizeof(double), dp = (size_t)sg.ldr * sizeof(double);
  const size_t hp = (size_t)ld_x * sizeof(double);
  if (stage && ld_x == rows && ld_y == sg.nymr && rows < sg.ldr) {
    const size_t nrow = (size_t)sg.nymr * sg.nzmr, bytes = nrow * w;
    if (to_dev) {
      AFID_CUDA(ctx, cudaMemcpyAsync(stage, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
      AFID_CUDA(ctx, launch_repack(ctx->stream, stage, rows, dev, sg.ldr, rows, nrow));
    } else {
      AFID_CUDA(ctx, launch_repack(ctx->stream, dev, sg.ldr, stage, rows, rows, nrow));
      AFID_CUDA(ctx, cudaMemcpyAsync(hdst, stage, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    }
    ctx->launches += 1;
    return AFID_OK;
  }
  for (int i = 0; i < sg.nzmr; ++i) {
    const size_t hoff = (size_t)i * ld_x * ld_y, doff = (size_t)i * sg.ldr * sg.nymr;
    if (to_dev)
      AFID_CUDA(ctx, cudaMemcpy2DAsync(dev + doff, dp, src + hoff, hp, w, sg.nymr, cudaMemcpyHostToDevice, ctx->stream));
    else
      AFID_CUDA(ctx, cudaMemcpy2DAsync(hdst + hoff, hp, dev + doff, dp, w, sg.nymr, cudaMemcpyDeviceToHost, ctx->stream));
  }
  return AFID_OK;
}

}  // namespace

extern "C" {

int afid_gpu_sal_create(afid_ctx_t *ctx, const afid_sal_grid_t *sg) {
  if (!ctx || !sg || ctx->sal) return AFID_E_INVALID;
  Geom &g = ctx->L.g;
  if (g.batch) return AFID_E_INVALID;
  const int nxmr = sg->nxmr, nymr = sg->nymr, nzmr = sg->nzmr;
  if (nxmr < 3 || nymr < 1 || nzmr < 1 || (g.nzm == 1) != (nzmr == 1)) return AFID_E_INVALID;
  const int MR = cn_choose_M(nxmr);
  if (MR < 0) return AFID_E_INVALID;
  if (!sg->xcr || !sg->udx3mr || !sg->g3rmr || !sg->ap3sskr || !sg->ac3sskr || !sg->am3sskr || !sg->salbp ||
      !sg->saltp || !(sg->pecs > 0.0))
    return AFID_E_INVALID;
  // every source row the kernels read stays inside the (wall-extended) columns
  // (x: inside the wall-extended source column; y/z: within two periods of the source grid)
  if (!stencil_ok(sg->to_ref[0], nxmr, -2, g.nxm - 2) || !stencil_ok(sg->to_ref[1], nymr, -2 * g.nym, 2 * g.nym) ||
      !stencil_ok(sg->to_ref[2], nzmr, -2 * g.nzm, 2 * g.nzm) || !stencil_ok(sg->to_coarse[0], g.nxm, -2, nxmr - 2) ||
      !stencil_ok(sg->to_coarse[1], g.nym, -2 * nymr, 2 * nymr) ||
      !stencil_ok(sg->to_coarse[2], g.nzm, -2 * nzmr, 2 * nzmr))
    return AFID_E_INVALID;
  const bool two_d = nzmr == 1;
  const size_t smem_step = sal_step_smem_bytes(MR, two_d);
  const size_t smem_ref = (size_t)4 * 3 * (g.nxm + 4) * sizeof(double);  // four warps' rows
  if (smem_step > 48 * 1024 || smem_ref > 227 * 1024) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  SalCtx *S = new (std::nothrow) SalCtx();
  if (!S) return AFID_E_ALLOC;
  SalGeom &q = S->sg;
  q.nxmr = nxmr;
  q.nymr = nymr;
  q.nzmr = nzmr;
  q.ldr = (nxmr + 1 + 7) / 8 * 8;
  q.ldu = (nxmr + 4 + 7) / 8 * 8;
  q.MR = MR;
  q.dxr = sg->dxr;
  q.dyr = sg->dyr;
  q.dzr = sg->dzr;
  q.udyr = 0.5 * sg->dyr;  // salinity.F90:279-283
  q.udzr = 0.5 * sg->dzr;
  q.udyrq = sg->dyr * sg->dyr / sg->pecs;
  q.udzrq = sg->dzr * sg->dzr / sg->pecs;
  q.lya = 1. / sg->dyr;  // InterpVelMgrd.F90:120, 204
  q.lza = 1. / sg->dzr;
  q.pecs = sg->pecs;
  q.sfixs = sg->sfixs;
  q.sfixn = sg->sfixn;
  S->active_s = sg->active_s;
  S->bycs = sg->bycs;
  S->relems = (size_t)q.ldr * nymr * nzmr;
  S->err = ctx->err;
  auto fail = [&](cudaError_t e) {
    delete S;
    return fail_cuda(ctx, e);
  };
  cudaError_t e = cudaSuccess;
  double **rf[8] = {&S->sal, &S->sal_o, &S->rusal, &S->vxr, &S->vyr, &S->vzr, &S->gyr, &S->gzr};
  for (double **p : rf)
    if ((e = dalloc(ctx, p, S->relems)) != cudaSuccess) return fail(e);
  double **cf[4] = {&S->gx, &S->gy, &S->gz, &S->salc};
  for (double **p : cf)
    if ((e = dalloc(ctx, p, ctx->field_elems)) != cudaSuccess) return fail(e);
  const size_t ntz = (size_t)3 * g.ldx * g.nym * nzmr, nu = (size_t)q.ldu * nymr * g.nzm;
  if ((e = dalloc(ctx, &S->tmp, std::max(ntz, nu))) != cudaSuccess) return fail(e);
  // 1-D tables
  std::vector<double> lxa(nxmr), tdxr(nxmr);
  for (int k = 0; k < nxmr; ++k) {
    lxa[k] = sg->xcr[k + 1] - sg->xcr[k];         // InterpVelMgrd.F90:53
    tdxr[k] = 0.5 * sg->dxr / sg->g3rmr[k];       // salinity.F90:605-607
  }
  auto up = [&](const double *h, size_t n, const double **d) -> cudaError_t {
    double *p = nullptr;
    cudaError_t r = dalloc(ctx, &p, n);
    if (r == cudaSuccess) r = cudaMemcpy(p, h, n * sizeof(double), cudaMemcpyHostToDevice);
    *d = p;
    return r;
  };
  SalTables &st = S->st;
  const size_t npl = (size_t)nymr * nzmr;
  if ((e = up(lxa.data(), nxmr, &st.lxa)) != cudaSuccess || (e = up(sg->udx3mr, nxmr, &st.udx3mr)) != cudaSuccess ||
      (e = up(tdxr.data(), nxmr, &st.tdxr)) != cudaSuccess || (e = up(sg->ap3sskr, nxmr, &st.ap)) != cudaSuccess ||
      (e = up(sg->ac3sskr, nxmr, &st.ac)) != cudaSuccess || (e = up(sg->am3sskr, nxmr, &st.am)) != cudaSuccess ||
      (e = up(sg->salbp, npl, &st.salbp)) != cudaSuccess || (e = up(sg->saltp, npl, &st.saltp)) != cudaSuccess)
    return fail(e);
  S->ap_d = st.ap;
  S->ac_d = st.ac;
  S->am_d = st.am;
  const afid_stencil_t *sts[6] = {&sg->to_ref[0], &sg->to_ref[1], &sg->to_ref[2],
                                  &sg->to_coarse[0], &sg->to_coarse[1], &sg->to_coarse[2]};
  for (int d = 0; d < 6; ++d) {
    int *pi = nullptr;
    if ((e = dalloc(ctx, &pi, (size_t)sts[d]->n)) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(pi, sts[d]->start, sts[d]->n * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail(e);
    st.st[d] = pi;
    if ((e = up(sts[d]->w, (size_t)4 * sts[d]->n, &st.w[d])) != cudaSuccess) return fail(e);
  }
  if ((e = dalloc(ctx, &S->cn_tab, cn_tab_doubles(MR, 1))) != cudaSuccess ||  // 3 substeps x 1 matrix
      (e = dalloc(ctx, &S->sc, 3)) != cudaSuccess || (e = dalloc(ctx, &S->red, 1)) != cudaSuccess)
    return fail(e);
  S->prof_blocks = sal_prof_blocks(q);
  if ((e = dalloc(ctx, &S->partial, (size_t)S->prof_blocks * 6 * nxmr)) != cudaSuccess ||
      (e = dalloc(ctx, &S->prof_out, (size_t)6 * nxmr)) != cudaSuccess)
    return fail(e);
  ctx->sal = S;
  g.salc = sg->active_s == 1 ? S->salc : nullptr;  // AddSalBuoyancy only for an active scalar
  g.bycs = sg->bycs;
  return AFID_OK;
}

int afid_gpu_sal_upload(afid_ctx_t *ctx, const double *sal, int ld_x, int ld_y) {
  if (!ctx || !ctx->sal || !sal) return AFID_E_INVALID;
  SalCtx &S = *ctx->sal;
  if (ld_x < S.sg.nxmr || ld_y < S.sg.nymr) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  int s;
  // sal_o holds no state between substeps: it stages the transfer
  if ((s = sal_copy(ctx, S.sal, S.sg.nxmr, sal, nullptr, ld_x, ld_y, true, S.sal_o)) != AFID_OK) return s;
  AFID_CUDA(ctx, cudaMemsetAsync(S.rusal, 0, S.relems * sizeof(double), ctx->stream));
  if ((s = sal_interp(ctx)) != AFID_OK) return s;  // main.F90:206-208
  return check_err_flag(ctx);
}

int afid_gpu_sal_download(afid_ctx_t *ctx, double *sal, int ld_x, int ld_y) {
  if (!ctx || !ctx->sal || !sal) return AFID_E_INVALID;
  SalCtx &S = *ctx->sal;
  if (ld_x < S.sg.nxmr || ld_y < S.sg.nymr) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  int s;
  if ((s = sal_copy(ctx, S.sal, S.sg.nxmr, nullptr, sal, ld_x, ld_y, false, S.sal_o)) != AFID_OK) return s;
  return check_err_flag(ctx);
}

int afid_gpu_sal_interpolate(afid_ctx_t *ctx) {
  if (!ctx || !ctx->sal) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  int s;
  if ((s = sal_interp(ctx)) != AFID_OK) return s;
  return check_err_flag(ctx);
}

int afid_gpu_sal_cfl(afid_ctx_t *ctx, double *cflmr) {
  if (!ctx || !ctx->sal || !cflmr) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  AFID_CUDA(ctx, timed(ctx, 8, [&] { return launch_sal_cfl(ctx->L, *ctx->sal); }));
  ctx->launches += 1;
  AFID_CUDA(ctx, cudaMemcpyAsync(ctx->host_scratch, ctx->sal->red, sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
  const int s = check_err_flag(ctx);
  const double v = ctx->host_scratch[0];
  *cflmr = (v != v) ? v : std::max(1.0e-8, v);  // CalcMaxCFL.F90:50; a NaN maximum is passed on
  return s;
}

int afid_gpu_sal_profiles(afid_ctx_t *ctx, double *out) {
  if (!ctx || !ctx->sal || !out) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  SalCtx &S = *ctx->sal;
  AFID_CUDA(ctx, timed(ctx, 8, [&] { return launch_sal_profiles(ctx->L, S, S.prof_out); }));
  ctx->launches += 2;
  AFID_CUDA(ctx, cudaMemcpyAsync(out, S.prof_out, (size_t)6 * S.sg.nxmr * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
  return check_err_flag(ctx);
}

int afid_gpu_sal_download_aux(afid_ctx_t *ctx, double *vxr, double *vyr, double *vzr, int ldr_x, int ldr_y,
                              double *salc, int ldc_x, int ldc_y) {
  if (!ctx || !ctx->sal) return AFID_E_INVALID;
  SalCtx &S = *ctx->sal;
  const Geom &g = ctx->L.g;
  if ((vxr || vyr || vzr) && (ldr_x < S.sg.nxmr + 1 || ldr_y < S.sg.nymr)) return AFID_E_INVALID;
  if (salc && (ldc_x < g.nxm || ldc_y < g.nym)) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  int s;
  if (vxr && (s = sal_copy(ctx, S.vxr, S.sg.nxmr + 1, nullptr, vxr, ldr_x, ldr_y, false)) != AFID_OK) return s;
  if (vyr && (s = sal_copy(ctx, S.vyr, S.sg.nxmr, nullptr, vyr, ldr_x, ldr_y, false)) != AFID_OK) return s;
  if (vzr && (s = sal_copy(ctx, S.vzr, S.sg.nxmr, nullptr, vzr, ldr_x, ldr_y, false)) != AFID_OK) return s;
  if (salc)
    for (int i = 0; i < g.nzm; ++i)
      AFID_CUDA(ctx, cudaMemcpy2DAsync(salc + (size_t)i * ldc_x * ldc_y, (size_t)ldc_x * sizeof(double),
                                       S.salc + (size_t)i * g.ldx * g.nym, (size_t)g.ldx * sizeof(double),
                                       (size_t)g.nxm * sizeof(double), g.nym, cudaMemcpyDeviceToHost, ctx->stream));
  return check_err_flag(ctx);
}

}  // extern "C"
