// serve.cu — the serving loop: tile requests queued by ppb_submit run on
// execution slots (one CUDA stream and buffer set each) as slots and HBM
// budget free up, so that tiles of different requests overlap on the device.
//
// Threads: one dispatcher and one worker per slot.  Slots keep the buffers,
// cuFFT plans and graphs of up to four grid sizes resident between requests.
// The dispatcher takes the oldest queued request, picks an idle slot (one
// that already holds the request's grid size first) and admits the request
// when the bytes held by all slots, plus the request's footprint if its slot
// does not hold that size yet, fit the context's HBM budget.  When memory is
// short, idle slots give up their least recently used sizes (then all their
// buffers); a request that does not fit with every other slot idle and empty
// fails with PPB_ERR_ADMISSION.  A worker runs run_tile_core on its slot,
// copies the records to host memory and marks the request done.  Results do
// not depend on which slot ran a request or on what ran beside it.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_map>

#include "ppb_ctx.h"

namespace ppb {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  ppb_tile_params p{};
  std::vector<double> Rf;
  uint64_t footprint = 0;
  Clock::time_point t_submit{}, t_done{};
  bool done = false;
  int32_t status = PPB_OK;
  std::string msg;
  std::vector<float> rec;
  int64_t count = 0, npeaks = 0;
  int32_t nf = 0;
  float RTHLmax = 0.f;
};

struct SlotState {
  std::unique_ptr<Slot> slot;
  std::thread th;
  std::shared_ptr<Request> job;   // the running request, null when idle
  uint64_t reserved = 0;          // bytes charged to this slot: what it holds, plus the
                                  // footprint of a new grid size while that runs
};

struct Server {
  ppb_ctx* ctx = nullptr;
  std::mutex mu;
  std::condition_variable cv_dispatch, cv_slot, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> reqs;
  std::vector<std::unique_ptr<SlotState>> slots;
  std::thread dispatcher;
  bool stop = false;
  uint64_t next_ticket = 1;
  uint64_t in_use = 0;
  // statistics
  std::vector<double> lat_ms;
  int64_t tiles_done = 0, peaks_done = 0, halos_done = 0, failed = 0;
  bool have_first = false;
  Clock::time_point t_first{}, t_last{};

  void dispatch_loop();
  void worker_loop(SlotState* st);
  void finish(const std::shared_ptr<Request>& r, Clock::time_point t);
};

void Server::finish(const std::shared_ptr<Request>& r, Clock::time_point t) {
  r->done = true;
  r->t_done = t;
  tiles_done++;
  if (r->status == PPB_OK) {
    peaks_done += r->npeaks;
    halos_done += r->count;
    lat_ms.push_back(std::chrono::duration<double, std::milli>(t - r->t_submit).count());
  } else {
    failed++;
  }
  t_last = t;
  cv_done.notify_all();
}

void Server::dispatch_loop() {
  std::unique_lock<std::mutex> lk(mu);
  const uint64_t budget = ctx->hbm_budget;
  while (true) {
    cv_dispatch.wait(lk, [&] { return stop || !queue.empty(); });
    if (stop) return;
    std::shared_ptr<Request> r = queue.front();
    const int n = r->p.n;
    SlotState* pick = nullptr;
    for (auto& s : slots)
      if (!s->job && s->slot->has_tile(n)) { pick = s.get(); break; }
    if (!pick)
      for (auto& s : slots)
        if (!s->job) { pick = s.get(); break; }
    if (!pick) {   // every slot busy: wait for one to finish
      cv_dispatch.wait(lk);
      continue;
    }
    // new bytes: the grid size's buffers unless resident, and the growth of
    // the slot's shell-stage buffers to this size's estimate
    const uint64_t sh_now = pick->slot->shell_bytes(), sh_est = shell_bytes_estimate(n);
    const uint64_t need = (pick->slot->has_tile(n) ? 0 : tile_bytes_estimate(n)) + (sh_est > sh_now ? sh_est - sh_now : 0);
    uint64_t after = in_use + need;
    // memory short: idle slots give up their least recently used grid sizes
    // (never the picked slot's copy of this request's size), then everything
    for (int pass = 0; pass < 2 && after > budget; pass++) {
      for (auto& s : slots) {
        if (s->job || after <= budget) continue;
        if (pass == 0) {
          for (int m = s->slot->lru_tile(s.get() == pick ? n : 0); m != 0 && after > budget;
               m = s->slot->lru_tile(s.get() == pick ? n : 0)) {
            const uint64_t freed = std::min<uint64_t>(s->slot->drop_tile(m), s->reserved);
            s->reserved -= freed;
            in_use -= freed;
            after -= std::min(after, freed);
          }
        } else if (s.get() != pick && s->reserved > 0) {
          s->slot->release_buffers();
          in_use -= s->reserved;
          after -= std::min(after, s->reserved);
          s->reserved = 0;
        }
      }
    }
    if (after > budget) {
      bool busy = false;
      for (auto& s : slots) busy = busy || (bool)s->job;
      if (busy) {   // wait for memory
        cv_dispatch.wait(lk);
        continue;
      }
      queue.pop_front();
      r->status = PPB_ERR_ADMISSION;
      r->msg = "request footprint (" + std::to_string(r->footprint >> 20) + " MiB) exceeds the HBM budget (" +
               std::to_string(budget >> 20) + " MiB)";
      finish(r, Clock::now());
      continue;
    }
    queue.pop_front();
    in_use += need;
    pick->reserved += need;
    pick->job = r;
    cv_slot.notify_all();
  }
}

void Server::worker_loop(SlotState* st) {
  cudaSetDevice(ctx->device);
  while (true) {
    std::shared_ptr<Request> r;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_slot.wait(lk, [&] { return stop || st->job; });
      if (stop) return;
      r = st->job;
    }
    int32_t status = PPB_OK;
    std::string msg;
    TileOut o;
    try {
      std::shared_lock<std::shared_mutex> rl(ctx->sh.mu);
      run_tile_core(ctx, *st->slot, &r->p, r->Rf.data(), (int)r->Rf.size(), &o);
      r->rec.resize((size_t)o.count * o.nfields);
      if (o.count > 0) copy_out(r->rec.data(), o.d_records, r->rec.size() * sizeof(float), st->slot->stream);
    } catch (const Error& e) {
      status = e.code;
      msg = e.msg;
    } catch (const std::exception& e) {
      status = PPB_ERR_INVALID;
      msg = e.what();
    } catch (...) {
      status = PPB_ERR_INVALID;
      msg = "unknown error";
    }
    std::lock_guard<std::mutex> lk(mu);
    r->status = status;
    r->msg = msg;
    r->count = o.count;
    r->npeaks = o.npeaks;
    r->nf = o.nfields;
    r->RTHLmax = o.RTHLmax;
    if (status == PPB_OK) {
      // keep the buffers for the next request of this grid size and charge
      // what the slot actually holds now
      const uint64_t held = st->slot->bytes_held();
      in_use = in_use - st->reserved + held;
      st->reserved = held;
    } else {
      st->slot->release_buffers();
      in_use -= st->reserved;
      st->reserved = 0;
    }
    st->job.reset();
    finish(r, Clock::now());
    cv_dispatch.notify_all();
  }
}

static Server& server_of(ppb_ctx* ctx) {
  if (!ctx->server) {
    auto sv = std::make_unique<Server>();
    sv->ctx = ctx;
    for (int i = 0; i < ctx->serve_slots; i++) {
      auto st = std::make_unique<SlotState>();
      st->slot = std::make_unique<Slot>();
      st->slot->init(ctx->device);
      sv->slots.push_back(std::move(st));
    }
    Server* raw = sv.get();
    for (auto& st : sv->slots) st->th = std::thread(&Server::worker_loop, raw, st.get());
    sv->dispatcher = std::thread(&Server::dispatch_loop, raw);
    ctx->server = std::move(sv);
  }
  return *ctx->server;
}

void server_stop(ppb_ctx* ctx) {
  if (!ctx->server) return;
  Server& sv = *ctx->server;
  {
    std::lock_guard<std::mutex> lk(sv.mu);
    sv.stop = true;
  }
  sv.cv_dispatch.notify_all();
  sv.cv_slot.notify_all();
  if (sv.dispatcher.joinable()) sv.dispatcher.join();
  for (auto& st : sv.slots)
    if (st->th.joinable()) st->th.join();
  ctx->server.reset();
}

}  // namespace ppb

using namespace ppb;

ppb_ctx::ppb_ctx() = default;

ppb_ctx::~ppb_ctx() {
  server_stop(this);
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
}

int64_t ppb_ctx::launches_total() const {
  int64_t t = sync.launches;
  if (server)
    for (const auto& st : server->slots) t += st->slot->launches;
  return t;
}

namespace ppb {
void graph_counts(const ppb_ctx* ctx, int64_t* out3) {
  out3[0] = ctx->sync.graph_launches;
  out3[1] = ctx->sync.graph_instantiations;
  out3[2] = ctx->sync.graph_updates;
  if (ctx->server)
    for (const auto& st : ctx->server->slots) {
      out3[0] += st->slot->graph_launches;
      out3[1] += st->slot->graph_instantiations;
      out3[2] += st->slot->graph_updates;
    }
}
}  // namespace ppb

extern "C" {

int32_t ppb_serve_config(ppb_ctx* ctx, int32_t slots) {
  if (!ctx || slots < 1 || slots > 32) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  if (ctx->server && (int)ctx->server->slots.size() != slots) {
    ctx->set_error("ppb_serve_config: the serving slots are already running");
    return PPB_ERR_INVALID;
  }
  ctx->serve_slots = slots;
  return PPB_OK;
}

int32_t ppb_submit(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int32_t nfilt, uint64_t* ticket) {
  if (!ctx || !ticket) return PPB_ERR_INVALID;
  try {
    check_params(p, Rf, nfilt);
    PPB_CUDA(cudaSetDevice(ctx->device));
    auto r = std::make_shared<Request>();
    r->p = *p;
    r->Rf.assign(Rf, Rf + nfilt);
    r->footprint = tile_footprint(p);
    r->t_submit = Clock::now();
    Server* sv;
    {
      std::lock_guard<std::recursive_mutex> lk(ctx->mu);
      sv = &server_of(ctx);
    }
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      r->ticket = sv->next_ticket++;
      if (!sv->have_first) {
        sv->have_first = true;
        sv->t_first = r->t_submit;
      }
      sv->reqs[r->ticket] = r;
      sv->queue.push_back(r);
      *ticket = r->ticket;
    }
    sv->cv_dispatch.notify_all();
    return PPB_OK;
  } catch (const Error& e) {
    ctx->set_error(e.msg);
    return e.code;
  } catch (...) {
    ctx->set_error("unknown error");
    return PPB_ERR_INVALID;
  }
}

int32_t ppb_wait(ppb_ctx* ctx, uint64_t ticket, int32_t timeout_ms, ppb_halo_buf* out) {
  if (!ctx || !out) return PPB_ERR_INVALID;
  Server* sv = ctx->server.get();
  if (!sv) return PPB_ERR_NOT_FOUND;
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return PPB_ERR_NOT_FOUND;
    r = it->second;
    if (timeout_ms < 0) {
      sv->cv_done.wait(lk, [&] { return r->done; });
    } else if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->done; })) {
      return PPB_ERR_TIMEOUT;
    }
    if (r->status != PPB_OK) {
      sv->reqs.erase(ticket);
      ctx->set_error(r->msg);
      return r->status;
    }
    out->nfields = r->nf;
    out->count = r->count;
    out->npeaks = r->npeaks;
    out->RTHLmax = r->RTHLmax;
    if (r->count > out->capacity) return PPB_ERR_CAPACITY;
    if (r->count > 0 && !out->records) {
      ctx->set_error("records buffer is null");
      return PPB_ERR_INVALID;
    }
    sv->reqs.erase(ticket);
  }
  const size_t bytes = r->rec.size() * sizeof(float);
  if (bytes == 0) return PPB_OK;
  if (is_device_ptr(out->records)) {
    if (cudaMemcpy(out->records, r->rec.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
      ctx->set_error("copying the records to the device buffer failed");
      return PPB_ERR_CUDA;
    }
  } else {
    std::memcpy(out->records, r->rec.data(), bytes);
  }
  return PPB_OK;
}

int32_t ppb_stats_get(ppb_ctx* ctx, ppb_stats* out) {
  if (!ctx || !out) return PPB_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  out->hbm_budget = ctx->hbm_budget;
  out->slots = ctx->serve_slots;
  Server* sv = ctx->server.get();
  if (!sv) return PPB_OK;
  std::lock_guard<std::mutex> lk(sv->mu);
  out->tiles_done = sv->tiles_done;
  out->peaks_done = sv->peaks_done;
  out->halos_done = sv->halos_done;
  out->failed = (int32_t)sv->failed;
  out->hbm_in_use = sv->in_use;
  out->queued = (int32_t)sv->queue.size();
  for (const auto& st : sv->slots) out->in_flight += st->job ? 1 : 0;
  if (!sv->lat_ms.empty()) {
    std::vector<double> l = sv->lat_ms;
    std::sort(l.begin(), l.end());
    auto q = [&](double f) {   // nearest-rank percentile
      size_t k = (size_t)std::ceil(f * (double)l.size());
      k = std::min(std::max<size_t>(k, 1), l.size());
      return l[k - 1];
    };
    out->p50_ms = q(0.50);
    out->p99_ms = q(0.99);
  }
  if (sv->have_first && sv->tiles_done > 0) {
    const double s = std::chrono::duration<double>(sv->t_last - sv->t_first).count();
    out->tiles_per_s = s > 0 ? (double)sv->tiles_done / s : 0.0;
  }
  return PPB_OK;
}

int32_t ppb_stats_reset(ppb_ctx* ctx) {
  if (!ctx) return PPB_ERR_INVALID;
  Server* sv = ctx->server.get();
  if (!sv) return PPB_OK;
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->lat_ms.clear();
  sv->tiles_done = sv->peaks_done = sv->halos_done = sv->failed = 0;
  sv->have_first = false;
  return PPB_OK;
}

}  // extern "C"
