// afid_serve.cpp — the request loop of include/afid_serve.h: pools of batches per size class,
// admission by device-memory footprint, chunked replay, harvest of finished slots.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <new>
#include <vector>

#include "afid_batch.h"
#include "afid_serve.h"
#include "afid_host_internal.h"

namespace {

// The inputs that decide which jobs can share a pool (afid_batch same-class rule).
struct ClassKey {
  int nxm, nym, nzm, istr3, nsst, active_t, gaxis, inslws, inslwn, tfixs, tfixn;
  double alx3, str3, xplusu, xminusu, dpdy;
  bool operator==(const ClassKey &o) const {
    return nxm == o.nxm && nym == o.nym && nzm == o.nzm && istr3 == o.istr3 && nsst == o.nsst &&
           active_t == o.active_t && gaxis == o.gaxis && inslws == o.inslws && inslwn == o.inslwn &&
           tfixs == o.tfixs && tfixn == o.tfixn && alx3 == o.alx3 && str3 == o.str3 && xplusu == o.xplusu &&
           xminusu == o.xminusu && dpdy == o.dpdy;
  }
};

ClassKey key_of(const afid_input_t &in) {
  ClassKey k{};
  k.nxm = in.nxm;
  k.nym = in.nym;
  k.nzm = in.nzm;
  k.istr3 = in.istr3;
  k.nsst = in.nsst;
  k.active_t = in.active_t;
  k.gaxis = in.gaxis;
  k.inslws = in.inslws;
  k.inslwn = in.inslwn;
  k.tfixs = in.tfixs;
  k.tfixn = in.tfixn;
  k.alx3 = in.alx3;
  k.str3 = in.str3;
  k.xplusu = in.xplusu;
  k.xminusu = in.xminusu;
  k.dpdy = in.dpdy;
  return k;
}

struct Job {
  afid_serve_job_t spec;
  double t_submit = 0.0, t_admit = 0.0;
  long long cells = 0;
  long long order = 0;  // submission number
  bool cancelled = false;  // afid_serve_cancel on a running job: finish at the next harvest
};

struct Pool {
  ClassKey key;
  afid_batch_t *b = nullptr;
  cudaStream_t stream = nullptr;
  int nslots = 0;
  std::vector<int> job;  // index into Server::running per slot, -1 = free
  std::vector<unsigned char> active;
  long long bytes = 0;
  long long cells_per_slot = 0;
  bool dirty = false;  // active flags changed since the last upload
  cudaEvent_t ev = nullptr;  // recorded after the pool's last chunk
  bool in_flight = false;    // a chunk is queued or running on the pool's stream
  long long launched = 0;    // pump launch order of that chunk
  int busy() const { return (int)std::count_if(job.begin(), job.end(), [](int j) { return j >= 0; }); }
};

}  // namespace

struct afid_server {
  afid_serve_config_t cfg{};
  std::chrono::steady_clock::time_point t0;
  std::deque<Job> queue;
  std::vector<Job> running;  // slots refer to entries here; freed entries are reused
  std::vector<int> free_running;
  std::vector<Pool *> pools;
  std::vector<afid_serve_result_t> done;
  long long submitted = 0;
  long long cells_in_flight = 0;
  long long cell_steps_done = 0;
  long long jobs_done = 0;
  long long launches = 0;  // chunks launched
  int pool_failures = 0;    // pools taken out after a failed operation (their jobs completed)
  int last_cuda_error = 0;  // the CUDA error seen at the last such failure, 0 if none
  int fail_test = 0;        // test hook: the fail_test-th next chunk launch counts as failed
  std::vector<afid_batch_stat_t> st;
  std::vector<double> nu, ke;
};

namespace {

double now_s(const afid_server_t *s) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

long long pool_bytes(const afid_server_t *s) {
  long long b = 0;
  for (const Pool *p : s->pools) b += p->bytes;
  return b;
}

void drop_pool(afid_server_t *s, size_t i) {
  Pool *p = s->pools[i];
  if (p->stream) cudaStreamSynchronize(p->stream);
  afid_batch_destroy(p->b);
  if (p->ev) cudaEventDestroy(p->ev);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
  s->pools.erase(s->pools.begin() + (long)i);
}

// A pool whose chunk, harvest or launch failed: its running jobs complete with `status` (their
// steps are not read back: the pool's state may not be), the pool is released and the server
// goes on with the others.  A CUDA error behind the failure is recorded and cleared, so a
// transient one does not stop later calls; a lasting one makes the next pools fail the same way.
void fail_pool(afid_server_t *s, Pool *p, int status) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) s->last_cuda_error = (int)e;
  for (int i = 0; i < p->nslots; ++i) {
    const int idx = p->job[i];
    if (idx < 0) continue;
    Job &j = s->running[idx];
    afid_serve_result_t r{};
    r.tag = j.spec.tag;
    r.errorcode = status;
    r.t_submit = j.t_submit;
    r.t_admit = j.t_admit;
    r.t_done = now_s(s);
    s->done.push_back(r);
    s->cells_in_flight -= j.cells;
    s->jobs_done += 1;
    p->job[i] = -1;
    j.cancelled = false;
    s->free_running.push_back(idx);
  }
  s->pool_failures += 1;
  for (size_t i = 0; i < s->pools.size(); ++i)
    if (s->pools[i] == p) {
      drop_pool(s, i);
      break;
    }
  cudaGetLastError();  // a failed synchronisation while releasing the pool is not carried on
}

// Create a pool for `in`'s class; AFID_E_CAPACITY when it does not fit the budget even after
// releasing idle pools of other classes.
int new_pool(afid_server_t *s, const afid_input_t &in, Pool **out) {
  const int nslots = in.nzm > 1 ? 1 : std::max(1, s->cfg.slots_per_pool);
  Pool *p = new (std::nothrow) Pool();
  if (!p) return AFID_E_ALLOC;
  p->key = key_of(in);
  int st = afid_batch_create(&in, nslots, s->cfg.precision, &p->b);
  if (st != AFID_OK) {
    delete p;
    return st;
  }
  p->bytes = afid_batch_device_bytes(p->b);
  // release idle pools while over budget
  while (pool_bytes(s) + p->bytes > s->cfg.hbm_budget_bytes) {
    size_t victim = s->pools.size();
    for (size_t i = 0; i < s->pools.size(); ++i)
      if (s->pools[i]->busy() == 0) {
        victim = i;
        break;
      }
    if (victim == s->pools.size()) {
      afid_batch_destroy(p->b);
      delete p;
      return AFID_E_CAPACITY;
    }
    drop_pool(s, victim);
  }
  if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->ev, cudaEventDisableTiming) != cudaSuccess ||
      afid_batch_set_stream(p->b, p->stream) != AFID_OK) {
    afid_batch_destroy(p->b);
    if (p->ev) cudaEventDestroy(p->ev);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
    return AFID_E_CUDA;
  }
  p->nslots = nslots;
  p->job.assign(nslots, -1);
  p->active.assign(nslots, 0);
  p->cells_per_slot = (long long)in.nxm * in.nym * in.nzm;
  s->pools.push_back(p);
  *out = p;
  return AFID_OK;
}

// Place job j into a free slot of its class (creating a pool if needed).  A pool whose chunk is
// still in flight takes no job (its slot set-up would wait for the chunk); kBusyPool
// then keeps the job queued until that pool is harvested.
constexpr int kBusyPool = -1;
int admit(afid_server_t *s, Job &j) {
  const ClassKey k = key_of(j.spec.in);
  Pool *pool = nullptr;
  int slot = -1;
  bool waiting = false;
  for (Pool *p : s->pools) {
    if (!(p->key == k)) continue;
    for (int i = 0; i < p->nslots; ++i)
      if (p->job[i] < 0) {
        if (p->in_flight) {
          waiting = true;
          break;
        }
        pool = p;
        slot = i;
        break;
      }
    if (pool) break;
  }
  if (!pool && waiting) return kBusyPool;
  if (!pool) {
    int st = new_pool(s, j.spec.in, &pool);
    if (st != AFID_OK) return st;
    slot = 0;
  }
  int st = afid_batch_configure(pool->b, slot, &j.spec.in);
  if (st == AFID_OK) st = afid_batch_seed(pool->b, slot, j.spec.seed);
  if (st == AFID_OK) st = afid_batch_set_limit(pool->b, slot, j.spec.nsteps);
  if (st != AFID_OK) return st;
  int idx;
  if (!s->free_running.empty()) {
    idx = s->free_running.back();
    s->free_running.pop_back();
  } else {
    idx = (int)s->running.size();
    s->running.emplace_back();
  }
  j.t_admit = now_s(s);
  s->running[idx] = j;
  pool->job[slot] = idx;
  pool->active[slot] = 1;
  pool->dirty = true;
  s->cells_in_flight += j.cells;
  return AFID_OK;
}

// Harvest one pool whose chunk has completed: results of the slots that reached their step
// count or stopped on an error code.
int harvest(afid_server_t *s, Pool *p) {
  p->in_flight = false;
  if (p->busy() == 0) return AFID_OK;
  s->st.resize(p->nslots);
  s->nu.resize(p->nslots);
  s->ke.resize(p->nslots);
  int st = afid_batch_stats(p->b, s->st.data(), s->nu.data(), s->ke.data());
  if (st != AFID_OK) return st;
  for (int i = 0; i < p->nslots; ++i) {
    const int idx = p->job[i];
    if (idx < 0) continue;
    Job &j = s->running[idx];
    const afid_batch_stat_t &x = s->st[i];
    if (x.ntime < j.spec.nsteps && x.errorcode == 0 && !j.cancelled) continue;
    if (j.spec.temp_out) {
      const int nx = j.spec.in.nxm + 1;
      st = afid_batch_download(p->b, i, nullptr, nullptr, nullptr, j.spec.temp_out, nullptr, nx, j.spec.in.nym);
      if (st != AFID_OK) return st;
    }
    afid_serve_result_t r{};
    r.tag = j.spec.tag;
    r.errorcode = j.cancelled ? AFID_E_CANCELLED : x.errorcode;
    r.steps_done = x.ntime;
    r.time = x.time;
    r.dt = x.dt;
    r.cfl = x.cfl;
    r.nu_vol = s->nu[i];
    r.ke = s->ke[i];
    r.t_submit = j.t_submit;
    r.t_admit = j.t_admit;
    r.t_done = now_s(s);
    s->done.push_back(r);
    s->cells_in_flight -= j.cells;
    s->cell_steps_done += j.cells * (long long)x.ntime;
    s->jobs_done += 1;
    p->job[i] = -1;
    p->active[i] = 0;
    p->dirty = true;
    j.cancelled = false;
    s->free_running.push_back(idx);
  }
  return AFID_OK;
}

bool has_cancelled(const afid_server_t *s, const Pool *p) {
  for (int idx : p->job)
    if (idx >= 0 && s->running[idx].cancelled) return true;
  return false;
}

// Device bytes of a pool's state arrays for a job of this input: nine FP64 field arrays (state
// and intermediates), four RK3 histories and phi at the explicit-term width, and the complex half
// spectrum (the layout afid_batch_create allocates; its 1-D tables and per-slot records come on
// top).  A lower bound of the pool's footprint.
long long pool_state_bytes(const afid_server_t *s, const afid_input_t &in) {
  const long long slots = in.nzm > 1 ? 1 : std::max(1, s->cfg.slots_per_pool);
  const long long planes = in.nzm > 1 ? in.nzm : slots;
  const long long ldx = (in.nxm + 1 + 7) / 8 * 8, ldxc = (in.nxm + 3) / 4 * 4;
  const long long tsz = s->cfg.precision == AFID_PREC_MIXED ? 4 : 8;
  const long long nf = ldx * in.nym * planes, nspec = ldxc * (in.nym / 2 + 1) * planes;
  return nf * (9 * 8 + 5 * tsz) + nspec * 2 * tsz;
}

}  // namespace

extern "C" {

int afid_serve_create(const afid_serve_config_t *cfg, afid_server_t **out) {
  return afid_guard([&]() -> int {
    if (!cfg || !out || cfg->hbm_budget_bytes <= 0 || cfg->chunk_steps < 1 ||
        (cfg->precision != AFID_PREC_FP64 && cfg->precision != AFID_PREC_MIXED))
      return AFID_E_INVALID;
    afid_server_t *s = new (std::nothrow) afid_server_t();
    if (!s) return AFID_E_ALLOC;
    s->cfg = *cfg;
    if (s->cfg.slots_per_pool < 1) s->cfg.slots_per_pool = 1;
    s->t0 = std::chrono::steady_clock::now();
    *out = s;
    return AFID_OK;
  });
}

int afid_serve_destroy(afid_server_t *s) {
  return afid_guard([&]() -> int {
    if (!s) return AFID_OK;
    while (!s->pools.empty()) drop_pool(s, s->pools.size() - 1);
    delete s;
    return AFID_OK;
  });
}

int afid_serve_submit(afid_server_t *s, const afid_serve_job_t *job) {
  return afid_guard([&]() -> int {
    if (!s || !job || job->nsteps < 1 || job->in.nxm < 2 || job->in.nym < 1 || job->in.nzm < 1 ||
        job->in.dpdz != 0.0 || job->in.flagsal)
      return AFID_E_INVALID;  // served jobs carry no salinity
    // a job whose pool cannot fit the budget even empty is refused here, not queued
    if (pool_state_bytes(s, job->in) > s->cfg.hbm_budget_bytes) return AFID_E_CAPACITY;
    Job j;
    j.spec = *job;
    j.t_submit = now_s(s);
    j.cells = (long long)job->in.nxm * job->in.nym * job->in.nzm;
    j.order = s->submitted++;
    s->queue.push_back(j);
    return AFID_OK;
  });
}

// One pass of the request loop, asynchronous per pool: pools whose chunk has completed are
// harvested, queued jobs are admitted into pools that are not running, and every idle pool with
// jobs gets its next chunk (each pool on its own stream, so a pool of small jobs does not wait
// for a pool of large ones).  When a pass finds nothing to do it waits for the oldest running
// chunk instead of spinning.
int afid_serve_pump(afid_server_t *s) {
  return afid_guard([&]() -> int {
    if (!s) return AFID_E_INVALID;
    bool progress = false;
    std::vector<std::pair<Pool *, int>> failed;  // taken out after each phase
    auto take_out = [&]() {
      for (auto &f : failed) fail_pool(s, f.first, f.second);
      if (!failed.empty()) progress = true;
      failed.clear();
    };
    // 1. harvest the pools whose chunk completed
    for (Pool *p : s->pools) {
      if (!p->in_flight) continue;
      const cudaError_t q = cudaEventQuery(p->ev);
      if (q == cudaErrorNotReady) continue;
      const int st = (q == cudaSuccess) ? harvest(s, p) : AFID_E_CUDA;
      if (st != AFID_OK) {
        p->in_flight = false;
        failed.emplace_back(p, st);
        continue;
      }
      progress = true;
    }
    take_out();
    // 2. admission in policy order
    std::vector<size_t> order(s->queue.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    const bool fifo = s->cfg.policy != AFID_SERVE_SHORTEST_FIRST;
    if (!fifo)
      std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        return (double)s->queue[a].cells * s->queue[a].spec.nsteps < (double)s->queue[b].cells * s->queue[b].spec.nsteps;
      });
    std::vector<char> taken(s->queue.size(), 0);
    for (size_t q : order) {
      Job &j = s->queue[q];
      if (s->cfg.max_cells_in_flight > 0 && s->cells_in_flight > 0 &&
          s->cells_in_flight + j.cells > s->cfg.max_cells_in_flight) {
        if (fifo) break;
        continue;
      }
      const int st = admit(s, j);
      if (st == kBusyPool) {  // its class's pool is running a chunk: retry after the harvest
        if (fifo) break;
        continue;
      }
      const bool no_room = (st == AFID_E_CAPACITY || st == AFID_E_ALLOC);
      if (no_room && !s->pools.empty()) {  // wait for running jobs to release memory
        if (fifo) break;
        continue;
      }
      if (st != AFID_OK) {
        // malformed, or larger than the whole budget: the job completes with the status
        afid_serve_result_t r{};
        r.tag = j.spec.tag;
        r.errorcode = st;
        r.t_submit = j.t_submit;
        r.t_admit = r.t_done = now_s(s);
        s->done.push_back(r);
      }
      taken[q] = 1;
      progress = true;
    }
    std::deque<Job> rest;
    for (size_t i = 0; i < s->queue.size(); ++i)
      if (!taken[i]) rest.push_back(s->queue[i]);
    s->queue.swap(rest);
    // 3. next chunk on every idle pool with running jobs (cancelled jobs leave first)
    for (Pool *p : s->pools) {
      if (p->in_flight || p->busy() == 0) continue;
      if (has_cancelled(s, p)) {
        const int hs = harvest(s, p);
        if (hs != AFID_OK) {
          failed.emplace_back(p, hs);
          continue;
        }
        progress = true;
        if (p->busy() == 0) continue;
      }
      int st = AFID_OK;
      if (p->dirty) {
        st = afid_batch_set_active(p->b, p->active.data());
        p->dirty = false;
      }
      if (st == AFID_OK && s->fail_test > 0 && --s->fail_test == 0) st = AFID_E_CUDA;  // test hook
      if (st == AFID_OK) st = afid_batch_step(p->b, s->cfg.chunk_steps);
      if (st == AFID_OK && cudaEventRecord(p->ev, p->stream) != cudaSuccess) st = AFID_E_CUDA;
      if (st != AFID_OK) {
        failed.emplace_back(p, st);
        continue;
      }
      p->in_flight = true;
      p->launched = s->launches++;
      progress = true;
    }
    take_out();
    // 4. nothing happened: wait for the oldest running chunk
    if (!progress) {
      Pool *oldest = nullptr;
      for (Pool *p : s->pools)
        if (p->in_flight && (!oldest || p->launched < oldest->launched)) oldest = p;
      if (oldest) {
        const int st = (cudaEventSynchronize(oldest->ev) == cudaSuccess) ? harvest(s, oldest) : AFID_E_CUDA;
        if (st != AFID_OK) {
          oldest->in_flight = false;
          fail_pool(s, oldest, st);
        }
      }
    }
    return AFID_OK;
  });
}

int afid_serve_cancel(afid_server_t *s, uint64_t tag) {
  return afid_guard([&]() -> int {
    if (!s) return AFID_E_INVALID;
    for (auto it = s->queue.begin(); it != s->queue.end(); ++it)
      if (it->spec.tag == tag) {
        afid_serve_result_t r{};
        r.tag = tag;
        r.errorcode = AFID_E_CANCELLED;
        r.t_submit = it->t_submit;
        r.t_admit = r.t_done = now_s(s);
        s->done.push_back(r);
        s->queue.erase(it);
        return AFID_OK;
      }
    for (const Pool *p : s->pools)
      for (int idx : p->job)
        if (idx >= 0 && s->running[idx].spec.tag == tag && !s->running[idx].cancelled) {
          s->running[idx].cancelled = true;  // finished at the pool's next harvest
          return AFID_OK;
        }
    return AFID_E_INVALID;
  });
}

int afid_serve_poll(afid_server_t *s, afid_serve_result_t *out, int max, int *n) {
  return afid_guard([&]() -> int {
    if (!s || !n || (max > 0 && !out)) return AFID_E_INVALID;
    const int k = std::min<int>(max, (int)s->done.size());
    for (int i = 0; i < k; ++i) out[i] = s->done[i];
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n = k;
    return AFID_OK;
  });
}

int afid_serve_status(const afid_server_t *s, afid_serve_status_t *st) {
  return afid_guard([&]() -> int {
    if (!s || !st) return AFID_E_INVALID;
    st->queued = (int)s->queue.size();
    st->running = 0;
    for (const Pool *p : s->pools) st->running += p->busy();
    st->pools = (int)s->pools.size();
    st->device_bytes = pool_bytes(s);
    st->cells_in_flight = s->cells_in_flight;
    st->cell_steps_done = s->cell_steps_done;
    st->jobs_done = s->jobs_done;
    st->pool_failures = s->pool_failures;
    st->last_cuda_error = s->last_cuda_error;
    return AFID_OK;
  });
}

double afid_serve_now(const afid_server_t *s) { return s ? now_s(s) : 0.0; }

int afid_serve_set_fail_test(afid_server_t *s, int nth) {
  if (!s || nth < 0) return AFID_E_INVALID;
  s->fail_test = nth;
  return AFID_OK;
}

}  // extern "C"
