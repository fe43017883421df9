// afid_batch.cu — batches of independent 2-D instances (include/afid_batch.h).
//
// A batch is one afid_ctx whose z index numbers the instances (Geom::batch): the substep
// kernels run every active instance in the same launches, each with its own scalars and CN
// tables.  The main-loop step control (CalcMaxCFL.F90:22-46, main.F90:287-304) runs per
// instance on the device, so one step is a fixed launch sequence, captured into a CUDA graph.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "afid_batch.h"
#include "afid_internal.h"

using namespace afid;

namespace {

// Step-control settings of one instance (bou.in IDTV DT CFLMAX DTMIN DTMAX).
struct InstCtl {
  double dt0, limit_cfl, dtmin, dtmax;
  int idtv;
};

// CFL of each active instance (CalcMaxCFL.F90:30-43): one warp per column, grid (chunks, slots).
__global__ void __launch_bounds__(256)
    k_batch_cfl(Geom g, Tables t, const double *__restrict__ vx, const double *__restrict__ vy,
                const double *__restrict__ vz, unsigned long long *__restrict__ out) {
  const int i = blockIdx.y;
  if (!inst_active(g, i)) return;
  bind_instance(g, i);
  const int lane = threadIdx.x & 31;
  double m = 0.0;
  for (int j = blockIdx.x * 8 + (threadIdx.x >> 5); j < g.nym; j += gridDim.x * 8) {
    const int jp = wrap_inc(j, g.nym);
    const size_t c = col_off(g, j, i), cjp = col_off(g, jp, i), cip = col_off(g, j, zinc(g, i));
    for (int k = lane; k < g.nxm; k += 32) {
      const double q = fabs((vz[c + k] + vz[cip + k]) * 0.5 * g.dz) + fabs((vy[c + k] + vy[cjp + k]) * 0.5 * g.dy) +
                       fabs((vx[c + k] + vx[c + k + 1]) * 0.5 * t.udx3m[k]);
      m = nan_max(m, q);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = nan_max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) atomicMax(out + i, (unsigned long long)__double_as_longlong(m));
}

// Maximum |div u| of each instance (CheckDivergence.F90:36-39), same layout as k_batch_cfl.
__global__ void __launch_bounds__(256)
    k_batch_div(Geom g, Tables t, const double *__restrict__ vx, const double *__restrict__ vy,
                const double *__restrict__ vz, unsigned long long *__restrict__ out) {
  const int i = blockIdx.y;
  bind_instance(g, i);
  const int lane = threadIdx.x & 31;
  double m = 0.0;
  for (int j = blockIdx.x * 8 + (threadIdx.x >> 5); j < g.nym; j += gridDim.x * 8) {
    const int jp = wrap_inc(j, g.nym);
    const size_t c = col_off(g, j, i), cjp = col_off(g, jp, i), cip = col_off(g, j, zinc(g, i));
    for (int k = lane; k < g.nxm; k += 32) {
      const double dq = (vz[cip + k] - vz[c + k]) * g.dz + (vy[cjp + k] - vy[c + k]) * g.dy +
                        (vx[c + k + 1] - vx[c + k]) * t.udx3m[k];
      m = nan_max(m, fabs(dq));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = nan_max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) atomicMax(out + i, (unsigned long long)__double_as_longlong(m));
}

// dt rule of main.F90:287-304 per instance.  An instance whose previous step raised an error
// code is switched off before this step (the reference exits after the step that set it).
__global__ void k_batch_dt(int nslots, unsigned char *__restrict__ active, const InstCtl *__restrict__ ctl,
                           const unsigned long long *__restrict__ cfl_bits, const int *__restrict__ ntime,
                           double *__restrict__ dt, double *__restrict__ cfl, int *__restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots || !active[i]) return;
  if (err[i] != 0) {
    active[i] = 0;
    return;
  }
  const double cflm = nan_max(0.00000001, __longlong_as_double((long long)cfl_bits[i]));  // CalcMaxCFL.F90:22
  const InstCtl c = ctl[i];
  double d = dt[i];
  if (c.idtv == 1) {
    if (ntime[i] > 1) {
      d = (cflm < 1.0e-8) ? c.dtmax : c.limit_cfl / cflm;
      if (d > c.dtmax) d = c.dtmax;
    }
    if (!(d >= c.dtmin)) err[i] = AFID_E_DTMIN;  // a NaN CFL gives a NaN dt: refused too
    cfl[i] = cflm;
  } else {
    if (!(cflm * d <= c.limit_cfl)) err[i] = AFID_E_CFL;
    cfl[i] = cflm * d;
  }
  dt[i] = d;
}

// time += dt (main.F90:313), step counter; a slot that reached its step limit switches off.
__global__ void k_batch_advance(int nslots, unsigned char *__restrict__ active, const double *__restrict__ dt,
                                double *__restrict__ time, int *__restrict__ ntime, const int *__restrict__ limit) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots || !active[i]) return;
  time[i] += dt[i];
  const int n = ntime[i] + 1;
  ntime[i] = n;
  if (limit[i] > 0 && n >= limit[i]) active[i] = 0;
}

// Volume sums of GlobalQuantities.F90:39-60 per instance: partial[(i*chunks + chunk)*3 + q].
__global__ void __launch_bounds__(256)
    k_batch_globals(Geom g, Tables t, const double *__restrict__ vx, const double *__restrict__ vy,
                    const double *__restrict__ vz, const double *__restrict__ temp, double *__restrict__ partial) {
  __shared__ double red[3][8];
  const int i = blockIdx.y;
  const int lane = threadIdx.x & 31;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int j = blockIdx.x * 8 + (threadIdx.x >> 5); j < g.nym; j += gridDim.x * 8) {
    const size_t c = col_off(g, j, i);
    for (int k = lane; k < g.nxm; k += 32) {
      const double fac2 = t.g3rc[k];
      const double vxcen = (vx[c + k] + vx[c + k + 1]) * 0.5;
      const double tc = temp[c + k];
      s0 += tc * vxcen * fac2;
      s1 += fac2 * (vz[c + k] * vz[c + k] + vy[c + k] * vy[c + k] + vx[c + k] * vx[c + k]);
      s2 += tc * fac2;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    red[0][threadIdx.x >> 5] = s0;
    red[1][threadIdx.x >> 5] = s1;
    red[2][threadIdx.x >> 5] = s2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int w = 0; w < 8; ++w) v += red[threadIdx.x][w];
    partial[((size_t)i * gridDim.x + blockIdx.x) * 3 + threadIdx.x] = v;
  }
}

__global__ void k_batch_gsum(const double *__restrict__ partial, int chunks, double *__restrict__ out) {
  const int i = blockIdx.x;
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int c = 0; c < chunks; ++c) v += partial[((size_t)i * chunks + c) * 3 + threadIdx.x];
    out[(size_t)i * 3 + threadIdx.x] = v;
  }
}

constexpr int kChunks = 4;  // blocks per instance in the per-instance reductions

}  // namespace

struct afid_batch {
  afid_ctx_t *ctx = nullptr;
  afid_input_t proto{};
  int nslots = 0;
  int precision = 0;
  bool three_d = false;  // one 3-D domain (nslots = 1) with the step control on the device
  int planes = 1;        // z planes per slot
  afid_tables_t *proto_tables = nullptr;
  std::vector<afid_input_t> cfg;
  std::vector<InstScal> inst_h;
  std::vector<InstCtl> ctl_h;
  std::vector<unsigned char> active_h;
  // device
  std::vector<void *> allocs;
  InstCtl *ctl = nullptr;
  double *dt = nullptr, *time = nullptr, *cfl = nullptr, *partial = nullptr, *gsum = nullptr;
  int *ntime = nullptr, *err = nullptr, *limit = nullptr;
  unsigned long long *cfl_bits = nullptr;
  double *host = nullptr;  // pinned staging for stats
  long long bytes = 0;
  // one captured step per temperature-buffer parity (the state alternates buffers each substep)
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double *graph_temp[2] = {nullptr, nullptr};
  long long launches_per_step = 0, launches = 0;
};

namespace {

template <typename T>
cudaError_t balloc(afid_batch_t *b, T **p, size_t n) {
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, (n ? n : 1) * sizeof(T));
  if (e != cudaSuccess) return e;
  b->allocs.push_back(q);
  b->bytes += (long long)((n ? n : 1) * sizeof(T));
  *p = static_cast<T *>(q);
  return cudaMemset(q, 0, (n ? n : 1) * sizeof(T));
}

// Inputs that must agree between the slots of one batch (sizes and wall-normal grid, the
// scheme and the boundary-condition switches); Ra, Pr, YLEN/ZLEN and the dt rule may differ.
bool same_class(const afid_input_t &a, const afid_input_t &p) {
  return a.nxm == p.nxm && a.nym == p.nym && a.nzm == p.nzm && a.alx3 == p.alx3 && a.istr3 == p.istr3 &&
         a.str3 == p.str3 && a.nsst == p.nsst && a.active_t == p.active_t && a.gaxis == p.gaxis &&
         a.inslws == p.inslws && a.inslwn == p.inslwn && a.tfixs == p.tfixs && a.tfixn == p.tfixn &&
         a.xplusu == p.xplusu && a.xminusu == p.xminusu && a.dpdy == p.dpdy && a.dpdz == 0.0;
}

void scal_ctl(const afid_input_t &in, const afid_params_t *p, InstScal *s, InstCtl *c) {
  s->dy = (double)in.nym / in.ylen;
  s->dyq = s->dy * s->dy;
  s->ren = p->ren;
  s->pect = p->pect;
  s->rren = 1.0 / p->ren;
  s->rpect = 1.0 / p->pect;
  s->udyq_re = s->dyq / p->ren;
  s->udyq_pe = s->dyq / p->pect;
  c->dt0 = in.dt;
  c->limit_cfl = in.limit_cfl;
  c->dtmin = in.dtmin;
  c->dtmax = in.dtmax;
  c->idtv = in.idtv;
}

// Scalars, wavenumbers and plates of one 2-D slot from its bou.in (ReadInputFile/CreateGrid/SetTempBCs).
int slot_tables(const afid_input_t &in, InstScal *s, std::vector<double> *ak2, std::vector<double> *bp,
                std::vector<double> *tp, InstCtl *c) {
  afid_tables_t *t = nullptr;
  int st = afid_tables_create(&in, AFID_PREC_FP64, &t);
  if (st != AFID_OK) return st;
  const afid_params_t *p = afid_tables_params(t);
  int n = 0;
  const double *a = afid_tables_array(t, "ak2", &n);
  ak2->assign(a, a + n);
  bp->assign(p->tempbp, p->tempbp + in.nym);
  tp->assign(p->temptp, p->temptp + in.nym);
  scal_ctl(in, p, s, c);
  afid_tables_destroy(t);
  return AFID_OK;
}

void drop_graphs(afid_batch_t *b) {
  for (int p = 0; p < 2; ++p) {
    if (b->graph[p]) cudaGraphExecDestroy(b->graph[p]);
    b->graph[p] = nullptr;
    b->graph_temp[p] = nullptr;
  }
}

int reset_slot(afid_batch_t *b, int slot) {
  afid_ctx_t *ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  const Geom &g = ctx->L.g;
  const size_t n = (size_t)g.ldx * g.nym * b->planes;
  const size_t tsz = ctx->L.mixed ? sizeof(float) : sizeof(double);
  for (void *r : {ctx->rux, ctx->ruy, ctx->ruz, ctx->rut})
    if (cudaMemsetAsync((char *)r + n * slot * tsz, 0, n * tsz, st) != cudaSuccess) return AFID_E_CUDA;
  const double dt0 = b->ctl_h[slot].dt0, zero = 0.0;
  const int izero = 0;
  if (cudaMemcpyAsync(b->dt + slot, &dt0, sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(b->time + slot, &zero, sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(b->ntime + slot, &izero, sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(b->err + slot, &izero, sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return AFID_E_CUDA;
  return cudaStreamSynchronize(st) == cudaSuccess ? AFID_OK : AFID_E_CUDA;
}

// Launch the sequence of one main-loop step (recorded into a graph by the caller).
int enqueue_step(afid_batch_t *b) {
  afid_ctx_t *ctx = b->ctx;
  const LaunchCtx &L = ctx->L;
  cudaStream_t st = ctx->stream;
  if (b->three_d) {
    if (launch_max_reduce(L, false, ctx->vx, ctx->vy, ctx->vz, b->cfl_bits) != cudaSuccess) return AFID_E_CUDA;
  } else {
    if (cudaMemsetAsync(b->cfl_bits, 0, sizeof(unsigned long long) * b->nslots, st) != cudaSuccess)
      return AFID_E_CUDA;
    k_batch_cfl<<<dim3(kChunks, b->nslots), 256, 0, st>>>(L.g, L.t, ctx->vx, ctx->vy, ctx->vz, b->cfl_bits);
  }
  k_batch_dt<<<(b->nslots + 127) / 128, 128, 0, st>>>(b->nslots, ctx->active_dev, b->ctl, b->cfl_bits, b->ntime,
                                                      b->dt, b->cfl, b->err);
  ctx->launches += 3;  // with k_batch_advance below
  if (cudaGetLastError() != cudaSuccess) return AFID_E_CUDA;
  int s = ctx_build_cn_batch(ctx, b->dt);
  for (int ns = 0; s == AFID_OK && ns < ctx->nsst; ++ns) s = ctx_run_substep(ctx, ns);
  if (s != AFID_OK) return s;
  k_batch_advance<<<(b->nslots + 127) / 128, 128, 0, st>>>(b->nslots, ctx->active_dev, b->dt, b->time, b->ntime,
                                                           b->limit);
  return cudaGetLastError() == cudaSuccess ? AFID_OK : AFID_E_CUDA;
}

// Copy one slot's fields between host (ld_x, ld_y, planes) and device (ldx, nym, planes).
int copy_slot(afid_batch_t *b, int slot, double *const dev[5], const double *const hsrc[5], double *const hdst[5],
              int ld_x, int ld_y) {
  afid_ctx_t *ctx = b->ctx;
  const Geom &g = ctx->L.g;
  const size_t plane = (size_t)g.ldx * g.nym, hplane = (size_t)ld_x * ld_y;
  const size_t dpitch = (size_t)g.ldx * sizeof(double), hpitch = (size_t)ld_x * sizeof(double);
  const size_t w = (size_t)g.nx * sizeof(double);
  const bool whole = (ld_y == g.nym);  // host planes back to back: one 2-D copy per field
  for (int f = 0; f < 5; ++f) {
    if (!(hsrc ? hsrc[f] : hdst[f])) continue;
    for (int p = 0; p < (whole ? 1 : b->planes); ++p) {
      double *d = dev[f] + plane * ((size_t)slot * b->planes + p);
      const size_t rows = whole ? (size_t)g.nym * b->planes : (size_t)g.nym;
      cudaError_t e = hsrc ? cudaMemcpy2DAsync(d, dpitch, hsrc[f] + hplane * p, hpitch, w, rows,
                                               cudaMemcpyHostToDevice, ctx->stream)
                           : cudaMemcpy2DAsync(hdst[f] + hplane * p, hpitch, d, dpitch, w, rows,
                                               cudaMemcpyDeviceToHost, ctx->stream);
      if (e != cudaSuccess) return ctx_fail(ctx, e);
    }
  }
  return AFID_OK;
}

}  // namespace

extern "C" {

int afid_batch_destroy(afid_batch_t *b) {
  if (!b) return AFID_OK;
  if (b->ctx) {
    cudaSetDevice(b->ctx->dev);
    cudaStreamSynchronize(b->ctx->stream);
  }
  drop_graphs(b);
  for (void *p : b->allocs) cudaFree(p);
  if (b->host) cudaFreeHost(b->host);
  if (b->ctx) afid_gpu_destroy(b->ctx);
  if (b->proto_tables) afid_tables_destroy(b->proto_tables);
  delete b;
  return AFID_OK;
}

int afid_batch_create(const afid_input_t *proto, int nslots, int precision, afid_batch_t **out) {
  if (!proto || !out || nslots < 1 || proto->nzm < 1 || proto->dpdz != 0.0) return AFID_E_INVALID;
  if (proto->nzm > 1 && nslots != 1) return AFID_E_INVALID;  // a 3-D domain is a batch of one
  if (proto->flagsal) return AFID_E_INVALID;                   // batches carry no salinity
  *out = nullptr;
  afid_batch_t *b = new (std::nothrow) afid_batch_t();
  if (!b) return AFID_E_ALLOC;
  b->proto = *proto;
  b->nslots = nslots;
  b->precision = precision;
  b->three_d = proto->nzm > 1;
  b->planes = proto->nzm;
  int s = afid_tables_create(proto, precision, &b->proto_tables);
  if (s != AFID_OK) {
    afid_batch_destroy(b);
    return s;
  }
  const int nym = proto->nym;
  InstScal sc{};
  InstCtl cc{};
  scal_ctl(*proto, afid_tables_params(b->proto_tables), &sc, &cc);
  b->cfg.assign(nslots, *proto);
  b->inst_h.assign(nslots, sc);
  b->ctl_h.assign(nslots, cc);
  b->active_h.assign(nslots, 0);
  afid_grid_t grid = *afid_tables_grid(b->proto_tables);
  afid_params_t prm = *afid_tables_params(b->proto_tables);
  prm.precision = precision;
  if (b->three_d) {
    s = ctx_create(&grid, &prm, nullptr, &b->ctx);
  } else {
    std::vector<double> ak2, bp, tp;
    if ((s = slot_tables(*proto, &sc, &ak2, &bp, &tp, &cc)) != AFID_OK || (int)ak2.size() < nym) {
      afid_batch_destroy(b);
      return s != AFID_OK ? s : AFID_E_INVALID;
    }
    std::vector<double> ak2_all((size_t)nslots * nym), bp_all((size_t)nslots * nym), tp_all((size_t)nslots * nym);
    for (int i = 0; i < nslots; ++i) {
      std::memcpy(&ak2_all[(size_t)i * nym], ak2.data(), nym * sizeof(double));
      std::memcpy(&bp_all[(size_t)i * nym], bp.data(), nym * sizeof(double));
      std::memcpy(&tp_all[(size_t)i * nym], tp.data(), nym * sizeof(double));
    }
    // The stacked geometry: z numbers the instances.
    grid.nzm = nslots;
    grid.zlen = (double)nslots;
    BatchSpec bs{nslots, b->inst_h.data(), ak2_all.data(), bp_all.data(), tp_all.data()};
    s = ctx_create(&grid, &prm, &bs, &b->ctx);
  }
  if (s != AFID_OK) {
    afid_batch_destroy(b);
    return s;
  }
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  if (b->three_d) {
    // device-side step control for the single domain: its scalars and one active flag
    afid_ctx_t *ctx = b->ctx;
    chk(balloc(b, &ctx->inst_dev, 1));
    chk(balloc(b, &ctx->active_dev, 1));
    if (e == cudaSuccess) e = cudaMemcpy(ctx->inst_dev, &sc, sizeof(InstScal), cudaMemcpyHostToDevice);
    ctx->ninst = 1;
    ctx->L.g.active = ctx->active_dev;
  } else {
    chk(cudaMemset(b->ctx->active_dev, 0, nslots));
  }
  chk(balloc(b, &b->ctl, nslots));
  chk(balloc(b, &b->dt, nslots));
  chk(balloc(b, &b->time, nslots));
  chk(balloc(b, &b->cfl, nslots));
  chk(balloc(b, &b->ntime, nslots));
  chk(balloc(b, &b->err, nslots));
  chk(balloc(b, &b->limit, nslots));
  chk(balloc(b, &b->cfl_bits, nslots));
  chk(balloc(b, &b->partial, (size_t)nslots * kChunks * 3));
  chk(balloc(b, &b->gsum, (size_t)nslots * 3));
  if (e == cudaSuccess) e = cudaMallocHost(&b->host, (size_t)nslots * 8 * sizeof(double));
  if (e == cudaSuccess)
    e = cudaMemcpy(b->ctl, b->ctl_h.data(), sizeof(InstCtl) * nslots, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    std::vector<double> dt0(nslots, cc.dt0);
    e = cudaMemcpy(b->dt, dt0.data(), sizeof(double) * nslots, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    afid_batch_destroy(b);
    return e == cudaErrorMemoryAllocation ? AFID_E_ALLOC : AFID_E_CUDA;
  }
  b->ctx->prof = false;  // event records would be captured into the step graph
  *out = b;
  return AFID_OK;
}

int afid_batch_set_stream(afid_batch_t *b, void *stream) {
  if (!b) return AFID_E_INVALID;
  return afid_gpu_set_stream(b->ctx, stream);
}

int afid_batch_configure(afid_batch_t *b, int slot, const afid_input_t *in) {
  if (!b || !in || slot < 0 || slot >= b->nslots || !same_class(*in, b->proto)) return AFID_E_INVALID;
  afid_ctx_t *ctx = b->ctx;
  cudaSetDevice(ctx->dev);
  InstScal sc{};
  InstCtl cc{};
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return AFID_E_CUDA;
  cudaError_t e = cudaSuccess;
  if (b->three_d) {
    // the domain's scalars are launch arguments: update them and re-capture the step
    afid_tables_t *t = nullptr;
    int s = afid_tables_create(in, b->precision, &t);
    if (s != AFID_OK) return s;
    afid_params_t prm = *afid_tables_params(t);
    prm.precision = b->precision;
    s = ctx_update_params(ctx, afid_tables_grid(t), &prm);
    scal_ctl(*in, &prm, &sc, &cc);
    afid_tables_destroy(t);
    if (s != AFID_OK) return s;
    drop_graphs(b);
    e = cudaMemcpy(ctx->inst_dev, &sc, sizeof(InstScal), cudaMemcpyHostToDevice);
  } else {
    std::vector<double> ak2, bp, tp;
    int s = slot_tables(*in, &sc, &ak2, &bp, &tp, &cc);
    if (s != AFID_OK) return s;
    const int nym = in->nym;
    if ((int)ak2.size() < nym) return AFID_E_INVALID;
    const Tables &t = ctx->L.t;
    const size_t off = (size_t)slot * nym;
    e = cudaMemcpy(ctx->inst_dev + slot, &sc, sizeof(InstScal), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(const_cast<double *>(t.ak2) + off, ak2.data(), nym * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(const_cast<double *>(t.tempbp) + off, bp.data(), nym * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(const_cast<double *>(t.temptp) + off, tp.data(), nym * sizeof(double), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMemcpy(b->ctl + slot, &cc, sizeof(InstCtl), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return ctx_fail(ctx, e);
  b->cfg[slot] = *in;
  b->inst_h[slot] = sc;
  b->ctl_h[slot] = cc;
  return AFID_OK;
}

int afid_batch_upload(afid_batch_t *b, int slot, const double *vx, const double *vy, const double *vz,
                      const double *temp, const double *pr, int ld_x, int ld_y) {
  if (!b || slot < 0 || slot >= b->nslots) return AFID_E_INVALID;
  afid_ctx_t *ctx = b->ctx;
  if (ld_x < ctx->L.g.nx || ld_y < ctx->L.g.nym) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  double *const dev[5] = {ctx->vx, ctx->vy, ctx->vz, ctx->temp, ctx->pr};
  const double *const src[5] = {vx, vy, vz, temp, pr};
  int s = copy_slot(b, slot, dev, src, nullptr, ld_x, ld_y);
  return s != AFID_OK ? s : reset_slot(b, slot);
}

int afid_batch_download(afid_batch_t *b, int slot, double *vx, double *vy, double *vz, double *temp,
                        double *pr, int ld_x, int ld_y) {
  if (!b || slot < 0 || slot >= b->nslots) return AFID_E_INVALID;
  afid_ctx_t *ctx = b->ctx;
  if (ld_x < ctx->L.g.nx || ld_y < ctx->L.g.nym) return AFID_E_INVALID;
  cudaSetDevice(ctx->dev);
  double *const dev[5] = {ctx->vx, ctx->vy, ctx->vz, ctx->temp, ctx->pr};
  double *const dst[5] = {vx, vy, vz, temp, pr};
  int s = copy_slot(b, slot, dev, nullptr, dst, ld_x, ld_y);
  return s != AFID_OK ? s : afid_batch_synchronize(b);
}

int afid_batch_seed(afid_batch_t *b, int slot, uint64_t seed) {
  if (!b || slot < 0 || slot >= b->nslots) return AFID_E_INVALID;
  afid_tables_t *t = nullptr;
  int s = afid_tables_create(&b->cfg[slot], AFID_PREC_FP64, &t);
  if (s != AFID_OK) return s;
  const int nx = b->proto.nxm + 1, nym = b->proto.nym;
  const size_t n = (size_t)nx * nym * b->planes;
  std::vector<double> temp(n, 0.0), zero(n, 0.0);
  s = afid_initial_temperature(t, seed, 1e-3, temp.data(), nx, nym);
  afid_tables_destroy(t);
  if (s != AFID_OK) return s;
  return afid_batch_upload(b, slot, zero.data(), zero.data(), zero.data(), temp.data(), zero.data(), nx, nym);
}

int afid_batch_set_limit(afid_batch_t *b, int slot, int nsteps) {
  if (!b || slot < 0 || slot >= b->nslots || nsteps < 0) return AFID_E_INVALID;
  afid_ctx_t *ctx = b->ctx;
  cudaSetDevice(ctx->dev);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpy(b->limit + slot, &nsteps, sizeof(int), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? AFID_OK : ctx_fail(ctx, e);
}

int afid_batch_set_active(afid_batch_t *b, const unsigned char *active) {
  if (!b || !active) return AFID_E_INVALID;
  afid_ctx_t *ctx = b->ctx;
  cudaSetDevice(ctx->dev);
  for (int i = 0; i < b->nslots; ++i) b->active_h[i] = active[i] ? 1 : 0;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpy(ctx->active_dev, b->active_h.data(), b->nslots, cudaMemcpyHostToDevice);
  return e == cudaSuccess ? AFID_OK : ctx_fail(ctx, e);
}

int afid_batch_step(afid_batch_t *b, int nsteps) {
  if (!b || nsteps < 0) return AFID_E_INVALID;
  afid_ctx_t *ctx = b->ctx;
  cudaSetDevice(ctx->dev);
  if (!ctx->tuned) {  // before the first capture: the tuner's launches must not be recorded
    const int s = ctx_autotune(ctx, false);
    if (s != AFID_OK) return s;
  }
  for (int n = 0; n < nsteps; ++n) {
    int p = (b->graph[0] && b->graph_temp[0] == ctx->temp) ? 0 : (b->graph[1] && b->graph_temp[1] == ctx->temp) ? 1 : -1;
    if (p < 0) {
      // Capture the step for this temperature-buffer parity.  The capture swaps the host-side
      // buffer pointers as the substeps do; they are put back, and swapped again below when
      // the replay is issued.
      p = b->graph[0] ? 1 : 0;
      double *temp0 = ctx->temp, *tempo0 = ctx->temp_o;
      const long long l0 = ctx->launches;
      cudaGraph_t graph = nullptr;
      cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return ctx_fail(ctx, e);
      int s = enqueue_step(b);
      e = cudaStreamEndCapture(ctx->stream, &graph);
      ctx->temp = temp0;
      ctx->temp_o = tempo0;
      if (s != AFID_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        ctx->launches = l0;
        return s != AFID_OK ? s : ctx_fail(ctx, e);
      }
      e = cudaGraphInstantiate(&b->graph[p], graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        b->graph[p] = nullptr;
        return ctx_fail(ctx, e);
      }
      b->graph_temp[p] = temp0;
      b->launches_per_step = ctx->launches - l0;
      ctx->launches = l0;
    }
    cudaError_t e = cudaGraphLaunch(b->graph[p], ctx->stream);
    if (e != cudaSuccess) return ctx_fail(ctx, e);
    for (int ns = 0; ns < ctx->nsst; ++ns) std::swap(ctx->temp, ctx->temp_o);
    b->launches += b->launches_per_step;
    ctx->launches += b->launches_per_step;
  }
  return AFID_OK;
}

int afid_batch_synchronize(afid_batch_t *b) {
  if (!b) return AFID_E_INVALID;
  return afid_gpu_synchronize(b->ctx);
}

int afid_batch_stats(afid_batch_t *b, afid_batch_stat_t *stats, double *nu_vol, double *ke) {
  if (!b) return AFID_E_INVALID;
  afid_ctx_t *ctx = b->ctx;
  cudaSetDevice(ctx->dev);
  const int n = b->nslots;
  cudaStream_t st = ctx->stream;
  const LaunchCtx &L = ctx->L;
  double *h = b->host;  // [dt | time | cfl | gsum(3) | ntime, err as ints]
  cudaError_t e = cudaSuccess;
  if (nu_vol || ke) {
    if (b->three_d) {
      e = launch_globals(L, ctx->vx, ctx->vy, ctx->vz, ctx->temp, ctx->partial, b->gsum);
    } else {
      k_batch_globals<<<dim3(kChunks, n), 256, 0, st>>>(L.g, L.t, ctx->vx, ctx->vy, ctx->vz, ctx->temp, b->partial);
      k_batch_gsum<<<n, 32, 0, st>>>(b->partial, kChunks, b->gsum);
      e = cudaGetLastError();
    }
    b->launches += 2;
    ctx->launches += 2;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h + 3 * (size_t)n, b->gsum, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, st);
  }
  int *hi = reinterpret_cast<int *>(h + 6 * (size_t)n);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, b->dt, n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h + n, b->time, n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h + 2 * (size_t)n, b->cfl, n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hi, b->ntime, n * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hi + n, b->err, n * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return ctx_fail(ctx, e);
  int s = afid_gpu_synchronize(ctx);
  if (s != AFID_OK) return s;
  // GlobalQuantities.F90:35,79,87-91
  const double vol = 1.0 / ((double)b->proto.nxm * (double)b->proto.nym * (double)b->planes);
  for (int i = 0; i < n; ++i) {
    if (stats) {
      stats[i].dt = h[i];
      stats[i].time = h[n + i];
      stats[i].cfl = h[2 * n + i];
      stats[i].ntime = hi[i];
      stats[i].errorcode = hi[n + i];
    }
    const double ra_pr = std::fabs(b->cfg[i].rayt) * b->cfg[i].prat;
    if (nu_vol) nu_vol[i] = 1.0 + std::sqrt(ra_pr) * h[3 * (size_t)n + 3 * i] * vol;
    if (ke) ke[i] = 0.5 * h[3 * (size_t)n + 3 * i + 1] * vol;
  }
  return AFID_OK;
}

int afid_batch_num_slots(const afid_batch_t *b) { return b ? b->nslots : 0; }

long long afid_batch_device_bytes(const afid_batch_t *b) { return b ? b->bytes + b->ctx->dev_bytes : 0; }

long long afid_batch_launch_count(const afid_batch_t *b) { return b ? b->launches : 0; }

int afid_batch_mean_profiles(afid_batch_t *b, int slot, double *out) {
  if (!b || !out || slot < 0 || slot >= b->nslots) return AFID_E_INVALID;
  afid_ctx_t *ctx = b->ctx;
  cudaSetDevice(ctx->dev);
  const Geom &g = ctx->L.g;
  const InstScal &sc = b->inst_h[slot];
  if (b->three_d)
    return ctx_mean_profiles(ctx, 0, g.nym * g.nzm, (double)g.nym * (double)g.nzm, g.ren, g.pect, out);
  return ctx_mean_profiles(ctx, slot * g.nym, g.nym, (double)g.nym, sc.ren, sc.pect, out);
}

int afid_batch_divmax(afid_batch_t *b, double *dmax) {
  if (!b || !dmax) return AFID_E_INVALID;
  afid_ctx_t *ctx = b->ctx;
  cudaSetDevice(ctx->dev);
  const LaunchCtx &L = ctx->L;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  if (b->three_d) {
    e = launch_max_reduce(L, true, ctx->vx, ctx->vy, ctx->vz, b->cfl_bits);
  } else {
    e = cudaMemsetAsync(b->cfl_bits, 0, sizeof(unsigned long long) * b->nslots, st);
    if (e == cudaSuccess) {
      k_batch_div<<<dim3(kChunks, b->nslots), 256, 0, st>>>(L.g, L.t, ctx->vx, ctx->vy, ctx->vz, b->cfl_bits);
      e = cudaGetLastError();
    }
  }
  b->launches += 1;
  ctx->launches += 1;
  std::vector<unsigned long long> h(b->nslots);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h.data(), b->cfl_bits, sizeof(unsigned long long) * b->nslots, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return ctx_fail(ctx, e);
  for (int i = 0; i < b->nslots; ++i) {
    double v;
    std::memcpy(&v, &h[i], sizeof(double));
    dmax[i] = v;
  }
  return AFID_OK;
}

int afid_batch_autotune(afid_batch_t *b, int force, afid_tune_info_t *info) {
  if (!b) return AFID_E_INVALID;
  cudaSetDevice(b->ctx->dev);
  if (cudaStreamSynchronize(b->ctx->stream) != cudaSuccess) return AFID_E_CUDA;
  const int s = ctx_autotune(b->ctx, force != 0);
  if (s == AFID_OK && force) drop_graphs(b);  // the captured step holds the old shape
  if (info) *info = b->ctx->tune;
  return s;
}

int afid_batch_set_k1_shape(afid_batch_t *b, int index) {
  if (!b) return AFID_E_INVALID;
  cudaSetDevice(b->ctx->dev);
  if (cudaStreamSynchronize(b->ctx->stream) != cudaSuccess) return AFID_E_CUDA;
  const int s = afid_gpu_set_k1_shape(b->ctx, index);
  if (s == AFID_OK) drop_graphs(b);  // the captured step holds the old shape
  return s;
}

}  // extern "C"
