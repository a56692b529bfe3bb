// ss3d_serve.cu -- serving form: a request loop over the simulation path.
//
// Requests (model, grid, seed, realization range, precision, output, optional
// conditioning data) arrive at any time through ss3d_server_submit.  A fixed
// number of slots, each a worker thread with its own CUDA stream and its own
// realization work space, take requests from one FIFO queue as soon as a slot
// is free and the request's device footprint fits the HBM budget: requests
// that arrive while others run are admitted as slots and memory free up, and
// their kernels overlap on the device (continuous batching).
//
//   footprint = growth of the slot's realization work space
//             + conditioning temporaries
//             + spectrum and its build temporaries when the model is not resident
//
// A slot keeps its work space between requests (taking it again costs nothing)
// up to retain_bytes; what it keeps stays charged to the budget.  When the head
// of the queue does not fit, an idle slot gives its work space back first.
//
// Spectra of models seen before stay resident in an LRU cache keyed by the
// model, grid and ipad; idle spectra are evicted when an admission needs the
// memory or when the cache exceeds its own budget.  A request whose spectrum
// is being built by another slot waits for that build instead of repeating it.
// When the head of the queue does not fit, later requests that fit may pass it,
// at most max_bypass times, so that a large request is never starved.  At most
// max_cond conditional requests run at once: their search and kriging kernels
// fill the GPU by themselves, and several of them only contend.
//
// The stages are the library's own entry points (ss3d_spectrum_create,
// ss3d_realize, ss3d_condition), so a request's result does not depend on what
// else runs: the same request alone and in a mix gives the same bits.  The
// reference runs one parameter file per process; this form has no counterpart.
//
// Dry-run mode (dry_run_ns_per_cell > 0) replaces the GPU stages by sleeps
// proportional to the work, with the same admission, cache and accounting, so
// the scheduler can be tested without a GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/specsim3d_gpu.h"
#include "ss3d_internal.h"

using namespace ss3d;

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  int64_t ticket = 0;
  std::vector<ss3d_struct> st;
  ss3d_request r{};           // copy of the caller's request; r.st points into st
  ss3d_cond_params cp{};
  bool cond = false;
  std::string key;            // spectrum cache key
  int64_t spec_bytes = 0;     // resident spectrum
  int64_t build_bytes = 0;    // temporaries of a spectrum build
  int64_t work_bytes = 0;     // realization work space (kept by the slot afterwards)
  int64_t tmp_bytes = 0;      // conditioning temporaries
  int64_t held = 0;           // transient bytes charged while the request runs
  int64_t cells = 0;
  int bypassed = 0;
  bool building = false;      // this request builds the spectrum
  double t_arrival = 0, t_submit = 0, t_admit = -1, t_done = -1;
  int status = SS3D_OK;
  int cache_hit = 0;
  bool done = false;
  std::string msg;
};

struct Entry {
  ss3d_spectrum* sp = nullptr;
  int64_t bytes = 0;
  int refs = 0;
  uint64_t last = 0;
  bool ready = false;
  int status = SS3D_OK;
  std::string msg;
};

std::string model_key(const ss3d_request& q) {
  std::string k;
  auto put = [&](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
  put(&q.nst, sizeof q.nst);
  for (int s = 0; s < q.nst; s++) {
    const ss3d_struct& t = q.st[s];
    put(&t.itype, sizeof t.itype);
    const double v[7] = {t.sill, t.ahmax, t.ahmin, t.avert, t.azimuth, t.dip, t.plunge};
    put(v, sizeof v);
  }
  put(&q.nugget, sizeof q.nugget);
  put(q.d, sizeof q.d);
  put(q.n, sizeof q.n);
  put(&q.ipad, sizeof q.ipad);
  return k;
}

}  // namespace

struct ss3d_server {
  ss3d_server_config cfg{};
  int dev = 0;
  bool dry = false;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Req*> queue;
  std::map<int64_t, Req*> reqs;      // submitted and not yet waited for
  std::map<std::string, Entry> cache;
  int64_t next_ticket = 1;
  int64_t charged = 0;               // running requests' temporaries + slots' work spaces
  int cond_running = 0;              // conditional requests on the GPU
  std::vector<int64_t> retained;     // work space kept by each slot
  int64_t cache_bytes = 0;           // bytes of resident (or building) spectra
  uint64_t tick = 0;
  bool stop = false;
  ss3d_serve_stats stats{};
  std::vector<std::thread> workers;
  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  int64_t budget() const { return cfg.hbm_budget; }
};

namespace {

void finish_locked(ss3d_server* s, Req* r, int status, const std::string& msg) {
  r->status = status;
  r->msg = msg;
  r->t_done = s->now();
  r->done = true;
  if (status == SS3D_OK) {
    s->stats.completed++;
    s->stats.cells += r->cells;
  } else {
    s->stats.failed++;
  }
}

// Idle spectra, least recently used first, evicted until `fits` holds; the
// handles go to `freed` and are released by the caller outside the lock.
template <class Fits>
void evict_locked(ss3d_server* s, const std::string& keep, std::vector<ss3d_spectrum*>& freed, Fits fits) {
  while (!fits()) {
    auto victim = s->cache.end();
    for (auto it = s->cache.begin(); it != s->cache.end(); ++it) {
      if (it->second.refs > 0 || !it->second.ready || it->first == keep) continue;
      if (victim == s->cache.end() || it->second.last < victim->second.last) victim = it;
    }
    if (victim == s->cache.end()) return;
    if (victim->second.sp) freed.push_back(victim->second.sp);
    s->cache_bytes -= victim->second.bytes;
    s->stats.evictions++;
    s->cache.erase(victim);
  }
}

// First admissible request of the queue for slot w, or nullptr.  Called with
// the lock.  *give_back is set when the head does not fit and slot w keeps a
// work space that would help.
Req* admit_locked(ss3d_server* s, int w, std::vector<ss3d_spectrum*>& freed, bool* give_back) {
  *give_back = false;
  for (size_t i = 0; i < s->queue.size(); ++i) {
    Req* r = s->queue[i];
    auto it = s->cache.find(r->key);
    const bool have = it != s->cache.end();
    const int64_t grow = std::max<int64_t>(0, r->work_bytes - s->retained[w]);
    const int64_t need = grow + r->tmp_bytes + (have ? 0 : r->spec_bytes + r->build_bytes);
    const int64_t alone = r->work_bytes + r->tmp_bytes + (have ? 0 : r->spec_bytes + r->build_bytes);
    if (alone > s->budget()) {
      s->queue.erase(s->queue.begin() + (long)i);
      finish_locked(s, r, SS3D_ENOMEM, "request needs " + std::to_string(alone) + " bytes of device memory, above "
                                           "the server's budget of " + std::to_string(s->budget()));
      s->cv.notify_all();
      --i;
      continue;
    }
    // conditional requests fill the GPU with their search and kriging
    // kernels: at most max_cond of them run at once, the other slots keep
    // serving unconditional requests beside them.  A head that waits only for
    // a conditional slot is not passed in the sense of max_bypass: requests
    // that take no such slot cannot delay it, so they are admitted past it
    // without limit (counting them stopped all admission, for as long as a
    // kriging call of the largest grids runs, once max_bypass was reached)
    if (r->cond && s->cond_running >= s->cfg.max_cond) continue;
    evict_locked(s, r->key, freed, [&] { return s->charged + s->cache_bytes + need <= s->budget(); });
    if (s->charged + s->cache_bytes + need <= s->budget()) {
      s->queue.erase(s->queue.begin() + (long)i);
      if (i > 0) {
        Req* h = s->queue.front();
        if (!(h->cond && s->cond_running >= s->cfg.max_cond)) h->bypassed++;
      }
      s->retained[w] += grow;
      r->held = r->tmp_bytes + (have ? 0 : r->build_bytes);
      s->charged += grow + r->held;
      if (have) {
        it->second.refs++;
        it->second.last = ++s->tick;
        r->cache_hit = 1;
        s->stats.cache_hits++;
      } else {
        Entry e;
        e.bytes = r->spec_bytes;
        e.refs = 1;
        e.last = ++s->tick;
        s->cache.emplace(r->key, e);
        s->cache_bytes += r->spec_bytes;
        r->building = true;
        s->stats.cache_misses++;
      }
      if (r->cond) s->cond_running++;
      r->t_admit = s->now();
      s->stats.peak_bytes = std::max(s->stats.peak_bytes, s->charged + s->cache_bytes);
      s->stats.peak_running = std::max<int64_t>(s->stats.peak_running, s->stats.running + 1);
      s->stats.running++;
      return r;
    }
    if (i == 0 && s->retained[w] > 0) *give_back = true;
    // the head does not fit: later requests may pass it a bounded number of times
    if (i == 0 && r->bypassed >= s->cfg.max_bypass) return nullptr;
  }
  return nullptr;
}

void release_spectra(std::vector<ss3d_spectrum*>& freed) {
  for (ss3d_spectrum* sp : freed) ss3d_spectrum_free(sp);
  freed.clear();
}

void sleep_ns(double ns) {
  if (ns > 0) std::this_thread::sleep_for(std::chrono::nanoseconds((long long)ns));
}

// The GPU work of one admitted request, outside the lock.
int run_request(ss3d_server* s, Req* r, std::string& msg) {
  const ss3d_request& q = r->r;
  ss3d_spectrum* sp = nullptr;
  int rc = SS3D_OK;
  if (r->building) {
    if (s->dry) {
      sleep_ns(s->cfg.dry_run_ns_per_cell * (double)r->spec_bytes / 12.0);
    } else {
      rc = ss3d_spectrum_create(q.st, q.nst, q.nugget, q.d, q.n, q.ipad, &sp, nullptr);
      if (rc) msg = ss3d_last_error();
    }
    std::lock_guard<std::mutex> lk(s->mu);
    Entry& e = s->cache[r->key];
    e.sp = sp;
    e.status = rc;
    e.msg = msg;
    e.ready = true;
    s->charged -= r->build_bytes;
    r->held -= r->build_bytes;
    s->cv.notify_all();
  } else {
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv.wait(lk, [&] { return s->cache[r->key].ready; });
    Entry& e = s->cache[r->key];
    sp = e.sp;
    rc = e.status;
    msg = e.msg;
  }
  if (rc) return rc;
  if (s->dry) {
    sleep_ns(s->cfg.dry_run_ns_per_cell * (double)r->cells);
    return SS3D_OK;
  }
  rc = ss3d_realize(sp, q.iseed, q.r_first, q.nreal, q.igauss, q.precision, q.out, q.out_dtype, nullptr);
  if (rc == SS3D_OK && r->cond) {
    ss3d_cond_stats cs{};
    rc = ss3d_condition(static_cast<double*>(q.out), q.n, q.nreal, q.xmin, q.d, q.st, q.nst, q.nugget, &r->cp, q.rows,
                        q.nrows, q.nvar, q.precision, &cs, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                        nullptr);
  }
  if (rc) msg = ss3d_last_error();
  return rc;
}

void worker_main(ss3d_server* s, int w) {
  // two streams per slot: unconditional requests at the highest priority,
  // conditional ones (long search and kriging kernels) at the lowest, so that
  // the block scheduler serves short requests between their blocks
  cudaStream_t st_hi = nullptr, st_lo = nullptr;
  if (!s->dry) {
    cudaSetDevice(s->dev);
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    cudaStreamCreateWithPriority(&st_hi, cudaStreamNonBlocking, hi);
    cudaStreamCreateWithPriority(&st_lo, cudaStreamNonBlocking, lo);
    ss3d_set_stream(st_hi);
  }
  std::vector<ss3d_spectrum*> freed;
  std::unique_lock<std::mutex> lk(s->mu);
  auto give_back_workspace = [&] {   // with the lock held; drops and retakes it
    const int64_t b = s->retained[w];
    lk.unlock();
    if (!s->dry) ss3d_release_workspace();   // on the slot's last stream, synchronised
    lk.lock();
    s->charged -= b;
    s->retained[w] = 0;
    s->cv.notify_all();
  };
  while (!s->stop) {
    bool give_back = false;
    Req* r = admit_locked(s, w, freed, &give_back);
    if (!freed.empty()) {
      lk.unlock();
      release_spectra(freed);
      lk.lock();
    }
    if (!r) {
      if (give_back) give_back_workspace();
      else s->cv.wait(lk);
      continue;
    }
    lk.unlock();
    std::string msg;
    if (!s->dry) ss3d_set_stream(r->cond ? st_lo : st_hi);
    const int rc = run_request(s, r, msg);
    lk.lock();
    s->charged -= r->held;
    r->held = 0;
    s->stats.running--;
    if (r->cond) s->cond_running--;
    auto it = s->cache.find(r->key);
    if (it != s->cache.end()) {
      it->second.refs--;
      it->second.last = ++s->tick;
      if (it->second.refs == 0 && it->second.status != SS3D_OK) {   // failed builds are not kept
        s->cache_bytes -= it->second.bytes;
        s->cache.erase(it);
      }
    }
    evict_locked(s, std::string(), freed, [&] { return s->cache_bytes <= s->cfg.cache_budget; });
    finish_locked(s, r, rc, msg);
    s->cv.notify_all();
    if (s->retained[w] > s->cfg.retain_bytes) give_back_workspace();
  }
  const int64_t b = s->retained[w];
  s->charged -= b;
  s->retained[w] = 0;
  lk.unlock();
  release_spectra(freed);
  if (!s->dry) {
    ss3d_set_stream(st_hi);
    ss3d_release_workspace();
    ss3d_set_stream(nullptr);
    cudaStreamDestroy(st_hi);
    cudaStreamDestroy(st_lo);
  }
}

}  // namespace

extern "C" int ss3d_server_create(const ss3d_server_config* cfg, ss3d_server** out) {
  if (!cfg || !out) return set_error(SS3D_EINVAL, "NULL argument");
  *out = nullptr;
  if (cfg->slots < 1 || cfg->slots > 64) return set_error(SS3D_EINVAL, "slots must be in 1..64");
  ss3d_server* s = new ss3d_server();
  s->cfg = *cfg;
  s->dry = cfg->dry_run_ns_per_cell > 0;
  s->t0 = Clock::now();
  if (!s->dry) {
    size_t fr = 0, tot = 0;
    if (cudaGetDevice(&s->dev) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      delete s;
      return set_error(SS3D_ECUDA, "server: no CUDA device");
    }
    if (s->cfg.hbm_budget <= 0) s->cfg.hbm_budget = (int64_t)(0.8 * (double)fr);
    // map pages into the stream-ordered pool now if asked: mapping pages while
    // requests run stalls the device for all of them (about a millisecond per
    // few MB)
    if (s->cfg.premap_bytes > 0)
      pool_premap((size_t)std::min<int64_t>(s->cfg.premap_bytes, s->cfg.hbm_budget));
    // load every kernel now: a kernel loaded on its first launch, while
    // requests run, may synchronise the device under all of them (a driver
    // without the loading entry points leaves the loads to the launches)
    if (ss3d_preload_kernels() != SS3D_OK) cudaGetLastError();
  } else if (s->cfg.hbm_budget <= 0) {
    delete s;
    return set_error(SS3D_EINVAL, "dry run needs an explicit hbm_budget");
  }
  if (s->cfg.retain_bytes <= 0)
    s->cfg.retain_bytes = std::min<int64_t>((int64_t)4 << 30, s->cfg.hbm_budget / (2 * s->cfg.slots));
  if (s->cfg.cache_budget <= 0) s->cfg.cache_budget = s->cfg.hbm_budget / 2;
  if (s->cfg.max_bypass <= 0) s->cfg.max_bypass = 16;
  if (s->cfg.max_cond <= 0) s->cfg.max_cond = 2;
  s->retained.assign(s->cfg.slots, 0);
  for (int w = 0; w < s->cfg.slots; w++) s->workers.emplace_back(worker_main, s, w);
  *out = s;
  return SS3D_OK;
}

extern "C" int ss3d_server_submit(ss3d_server* s, const ss3d_request* q, int64_t* ticket) {
  if (!s || !q || !ticket) return set_error(SS3D_EINVAL, "NULL argument");
  if (!q->st || q->nst < 1 || q->nst > MAXST) return set_error(SS3D_EINVAL, "nst must be in 1..10");
  if (q->n[0] < 1 || q->n[1] < 1 || q->n[2] < 1) return set_error(SS3D_EINVAL, "grid sizes must be positive");
  if (q->nreal < 1 || q->r_first < 0) return set_error(SS3D_EINVAL, "nreal must be >= 1 and r_first >= 0");
  if (q->igauss != 0 && q->igauss != 1) return set_error(SS3D_EINVAL, "igauss must be 0 or 1");
  if (q->precision != SS3D_FP64 && q->precision != SS3D_FP32) return set_error(SS3D_EINVAL, "unknown precision");
  if (q->out_dtype != SS3D_OUT_F32 && q->out_dtype != SS3D_OUT_F64) return set_error(SS3D_EINVAL, "unknown out_dtype");
  if (!q->out && !s->dry) return set_error(SS3D_EINVAL, "out is NULL");
  const bool cond = q->nrows > 0;
  if (cond && (!q->cp || !q->rows || q->nvar < 1 || q->out_dtype != SS3D_OUT_F64))
    return set_error(SS3D_EINVAL, "conditional requests need cp, rows, nvar and a float64 output");
  int np[3];
  if (int rc = ss3d_grid_size(q->st, q->nst, q->d, q->n, q->ipad, np)) return rc;
  bool host_out = false;
  if (!s->dry) {
    // rejected at submission, not when a slot reaches the request: device
    // output on another device, or not aligned for the row stores
    bool dev_out = false;
    const size_t oel = q->out_dtype == SS3D_OUT_F32 ? 4 : 8;
    if (int rc = check_ptr(q->out, s->dev, (q->n[0] % 2 == 0 ? 2 : 1) * oel, "out", &dev_out)) return rc;
    host_out = !dev_out;
  }
  Req* r = new Req();
  r->st.assign(q->st, q->st + q->nst);
  r->r = *q;
  r->r.st = r->st.data();
  r->cond = cond;
  if (cond) {
    r->cp = *q->cp;
    r->r.cp = &r->cp;
  }
  r->key = model_key(r->r);
  const int64_t H = np[0] >= 2 ? np[0] / 2 + 1 : 1, HP = (H + 1) & ~(int64_t)1;
  const int64_t nh = (int64_t)np[2] * np[1] * HP;
  const int64_t M = (int64_t)q->n[0] * q->n[1] * q->n[2];
  r->spec_bytes = nh * (int64_t)(sizeof(double) + sizeof(float)) + (1 << 20);
  r->build_bytes = nh * (int64_t)(2 * sizeof(double)) + (1 << 20);
  r->work_bytes = realize_bytes_for(np, q->n, q->nreal, q->precision, host_out ? 1 : 0);
  if (cond) {
    const int64_t per_node = 4LL * q->cp->ndmax + 4;
    r->tmp_bytes = (host_out ? M * q->nreal * 8 : 0) + std::min<int64_t>(M, ((int64_t)1 << 30) / per_node) * per_node +
                   (int64_t)q->nrows * (8LL * q->nreal + 96) + (1 << 20);
  }
  r->cells = M * q->nreal;
  std::lock_guard<std::mutex> lk(s->mu);
  r->t_submit = s->now();
  r->t_arrival = q->t_arrival >= 0 ? q->t_arrival : r->t_submit;
  r->ticket = s->next_ticket++;
  s->reqs[r->ticket] = r;
  s->queue.push_back(r);
  s->stats.submitted++;
  *ticket = r->ticket;
  s->cv.notify_all();
  return SS3D_OK;
}

extern "C" int ss3d_server_wait(ss3d_server* s, int64_t ticket, ss3d_result* res) {
  if (!s) return set_error(SS3D_EINVAL, "server is NULL");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return set_error(SS3D_EINVAL, "unknown ticket");
  Req* r = it->second;
  s->cv.wait(lk, [&] { return r->done; });
  s->reqs.erase(it);
  lk.unlock();
  if (res) {
    res->status = r->status;
    res->cache_hit = r->cache_hit;
    res->t_arrival = r->t_arrival;
    res->t_submit = r->t_submit;
    res->t_admit = r->t_admit;
    res->t_done = r->t_done;
    res->footprint = r->work_bytes + r->tmp_bytes + (r->building ? r->spec_bytes + r->build_bytes : 0);
  }
  const int rc = r->status;
  const std::string msg = r->msg;
  delete r;
  if (rc) return set_error(rc, msg.c_str());
  return SS3D_OK;
}

extern "C" int ss3d_server_stats(ss3d_server* s, ss3d_serve_stats* out) {
  if (!s || !out) return set_error(SS3D_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->queued = (int64_t)s->queue.size();
  out->cached_spectra = (int64_t)s->cache.size();
  out->cache_bytes = s->cache_bytes;
  out->charged_bytes = s->charged;
  out->budget_bytes = s->cfg.hbm_budget;
  return SS3D_OK;
}

extern "C" double ss3d_server_clock(ss3d_server* s) { return s ? s->now() : 0.0; }

extern "C" void ss3d_server_free(ss3d_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (Req* r : s->queue) finish_locked(s, r, SS3D_EINVAL, "server stopped before the request ran");
    s->queue.clear();
    s->cv.notify_all();
  }
  for (std::thread& t : s->workers) t.join();
  for (auto& kv : s->cache)
    if (kv.second.sp) ss3d_spectrum_free(kv.second.sp);
  for (auto& kv : s->reqs) delete kv.second;
  delete s;
}
