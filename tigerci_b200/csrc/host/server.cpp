// Continuously batched CI-solve server on one GPU (tci_server_*).
//
// The reference solves one CI problem per process (tiger_ci.f90 drives one
// davidson_liu).  A serving deployment instead receives a stream of solves of
// different sizes (potential-energy-surface points, several roots each).  This
// server keeps up to `slots` of them on the GPU at once:
//
//   submit -> planners (host threads: CSF space + sigma plan, the request's
//             device-memory estimate) -> ready queue (FIFO) -> admission
//             (a free slot and room in the HBM budget) -> worker: device
//             context on its own CUDA stream, device-resident Davidson,
//             context released -> result
//
// A request's Cholesky vectors, operators and Davidson subspace stay in HBM
// for the whole solve; the sigma builds of the admitted requests run on
// separate streams and overlap on the device.  Requests that arrive while
// others run are planned on the host in the meantime and admitted as soon as a
// slot and memory free up.  Every request is solved by the same deterministic
// kernels as a lone tci_davidson call, so its result does not depend on what
// else runs beside it.
//
// Failure handling, all on the host: a request whose estimate exceeds the
// whole budget is rejected (TCI_ERR_MEMORY); non-finite operator input is
// rejected at submission (TCI_ERR_INPUT); a request can be cancelled while
// queued or mid-solve (TCI_ERR_CANCELLED, the solver polls a flag between
// iterations); a worker thread that dies is detected by a supervisor thread,
// which re-queues its request and starts a replacement worker.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/tigerci_sigma.h"
#include "capi_internal.h"
#include "plan.h"

using namespace tci;

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { RQ_PLAN, RQ_READY, RQ_RUNNING, RQ_DONE };

struct Request {
  int64_t id = 0;
  // owned copies of the caller's inputs (the caller may free them after submit)
  tci_deck deck{};
  std::vector<int64_t> ref_occ, nm1p, nm1i, nm2p, nm2i;
  std::vector<double> h, chol;
  int64_t nchol = 0;
  double core_energy = 0;
  int64_t nroots = 1, maxit = 0;
  double tol_r = 1e-6, tol_e = 1e-6;
  // pipeline
  ReqState state = RQ_PLAN;
  std::unique_ptr<CsfSpace> sp;
  std::unique_ptr<Plan> plan;
  int64_t total_csfs = 0;
  int64_t subspace_bytes = 0;
  double est_bytes = 0;
  int32_t cancel = 0;  // read by the solver with an atomic load
  int status = TCI_OK;
  std::string error;
  std::vector<double> energies;
  int64_t iterations = 0;
  double t_submit = 0, t_planned = -1, t_admitted = -1, t_done = -1;

  tci_operator op() const { return tci_operator{h.data(), chol.data(), nchol, core_energy}; }
};

// Thrown inside a worker by the fault injector: the worker thread ends with
// its request still assigned, as if it had died.
struct WorkerDeath {};

}  // namespace

struct tci_server {
  tci_server_config cfg{};
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv;
  std::map<int64_t, std::shared_ptr<Request>> reqs;
  std::deque<std::shared_ptr<Request>> to_plan, ready;
  std::vector<std::shared_ptr<Request>> slot_req;  // request held by each worker slot
  std::vector<char> slot_dead;
  std::vector<std::thread> workers, planners;
  std::thread supervisor;
  double reserved = 0, peak_reserved = 0;
  int running = 0, peak_running = 0;
  int64_t next_id = 1, admissions = 0, worker_restarts = 0;
  int64_t n_ok = 0, n_failed = 0, n_cancelled = 0;
  double first_submit = -1, last_done = -1;
  std::vector<double> tts;  // time to solution of successful requests
  bool stopping = false;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

  void finish(const std::shared_ptr<Request>& r, int status, const std::string& err) {
    // caller holds mu
    r->status = status;
    r->error = err;
    r->t_done = now();
    r->state = RQ_DONE;
    r->sp.reset();
    r->plan.reset();
    r->h.clear();
    r->h.shrink_to_fit();
    r->chol.clear();
    r->chol.shrink_to_fit();
    if (status == TCI_OK) {
      n_ok++;
      tts.push_back(r->t_done - r->t_submit);
      last_done = std::max(last_done, r->t_done);
    } else if (status == TCI_ERR_CANCELLED) {
      n_cancelled++;
    } else {
      n_failed++;
    }
    cv.notify_all();
  }

  void planner_loop() {
    for (;;) {
      std::shared_ptr<Request> r;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stopping || !to_plan.empty(); });
        if (stopping) return;
        r = to_plan.front();
        to_plan.pop_front();
      }
      int status = TCI_OK;
      std::string err;
      auto sp = std::make_unique<CsfSpace>();
      auto plan = std::make_unique<Plan>();
      try {
        build_space_from_c(&r->deck, *sp);
        Operator o;
        const tci_operator cop = r->op();
        operator_from_c(&cop, *sp, o);
        build_plan(*sp, o, *plan);
      } catch (...) {
        status = guard_status(std::current_exception());
        char buf[512];
        tci_last_error(buf, sizeof(buf));
        err = buf;
      }
      std::lock_guard<std::mutex> lk(mu);
      if (r->state == RQ_DONE) continue;  // cancelled while planning
      if (status != TCI_OK) {
        finish(r, status, err);
        continue;
      }
      r->total_csfs = plan->total_csfs;
      const int64_t per_root = cfg.subspace_vectors_per_root > 0 ? cfg.subspace_vectors_per_root : 12;
      r->subspace_bytes = 16 * r->total_csfs * per_root * r->nroots;
      double peak = 0, resident = 0;
      ctx_device_bytes(*plan, cfg.precision, &peak, &resident);
      const double dav = (double)tci_davidson_bytes(r->total_csfs, r->nroots, r->maxit, r->subspace_bytes);
      r->est_bytes = std::max(peak, resident + dav);
      if (r->est_bytes > (double)cfg.hbm_budget_bytes) {
        finish(r, TCI_ERR_MEMORY,
               "request needs " + std::to_string((long long)r->est_bytes) + " device bytes, more than the HBM budget");
        continue;
      }
      r->sp = std::move(sp);
      r->plan = std::move(plan);
      r->t_planned = now();
      r->state = RQ_READY;
      // planned requests queue by arrival; planning order does not matter
      auto pos = std::find_if(ready.begin(), ready.end(), [&](const std::shared_ptr<Request>& q) { return q->id > r->id; });
      ready.insert(pos, r);
      cv.notify_all();
    }
  }

  void worker_loop(int slot) {
    try {
      for (;;) {
        std::shared_ptr<Request> r;
        {
          std::unique_lock<std::mutex> lk(mu);
          // strict FIFO admission: the head of the ready queue waits for room
          cv.wait(lk, [&] {
            return stopping || (!ready.empty() && reserved + ready.front()->est_bytes <= (double)cfg.hbm_budget_bytes);
          });
          if (stopping) return;
          r = ready.front();
          ready.pop_front();
          r->state = RQ_RUNNING;
          r->t_admitted = now();
          reserved += r->est_bytes;
          peak_reserved = std::max(peak_reserved, reserved);
          running++;
          peak_running = std::max(peak_running, running);
          slot_req[slot] = r;
          admissions++;
          if (cfg.inject_worker_exit_at > 0 && admissions == cfg.inject_worker_exit_at) throw WorkerDeath{};
        }
        int status = TCI_OK;
        std::string err;
        std::vector<double> e(r->nroots, std::nan(""));
        int64_t iters = 0;
        if (cfg.schedule_only) {
          // scheduling run: hold the slot and the reservation, no device work
          const auto until = Clock::now() + std::chrono::duration<double, std::milli>(cfg.schedule_only_ms);
          while (Clock::now() < until && __atomic_load_n(&r->cancel, __ATOMIC_ACQUIRE) == 0)
            std::this_thread::sleep_for(std::chrono::milliseconds(1));
          if (__atomic_load_n(&r->cancel, __ATOMIC_ACQUIRE) != 0) status = TCI_ERR_CANCELLED;
        } else {
          tci_ctx* ctx = nullptr;
          status = ctx_from_plan(std::move(*r->sp), std::move(*r->plan), r->chol.data(), cfg.device, cfg.precision,
                                 128, &ctx);
          if (status == TCI_OK) ctx_set_tc_gemms(ctx, cfg.tc_gemms);
          if (status == TCI_OK)
            status = tci_davidson_ex(ctx, r->nroots, r->tol_r, r->tol_e, r->maxit, r->subspace_bytes, &r->cancel,
                                     e.data(), nullptr, &iters);
          if (status != TCI_OK) {
            char buf[512];
            tci_last_error(buf, sizeof(buf));
            err = buf;
          }
          tci_destroy(ctx);
        }
        std::lock_guard<std::mutex> lk(mu);
        reserved -= r->est_bytes;
        running--;
        slot_req[slot].reset();
        r->energies = e;
        r->iterations = iters;
        finish(r, status, err);
      }
    } catch (const WorkerDeath&) {
      std::lock_guard<std::mutex> lk(mu);
      slot_dead[slot] = 1;
      cv.notify_all();
    }
  }

  // Restarts dead workers and puts their requests back at the head of the queue.
  void supervisor_loop() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      cv.wait(lk, [&] {
        return stopping || std::any_of(slot_dead.begin(), slot_dead.end(), [](char d) { return d != 0; });
      });
      if (stopping) return;
      for (size_t s = 0; s < slot_dead.size(); ++s) {
        if (!slot_dead[s]) continue;
        std::thread old = std::move(workers[s]);
        lk.unlock();
        if (old.joinable()) old.join();
        lk.lock();
        std::shared_ptr<Request> r = slot_req[s];
        slot_req[s].reset();
        if (r && r->state == RQ_RUNNING) {
          reserved -= r->est_bytes;
          running--;
          r->state = RQ_READY;
          r->t_admitted = -1;
          ready.push_front(r);
        }
        slot_dead[s] = 0;
        worker_restarts++;
        workers[s] = std::thread([this, s] { worker_loop((int)s); });
        cv.notify_all();
      }
    }
  }
};

namespace {

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return std::nan("");
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);
  const size_t i = (size_t)std::floor(pos);
  const double f = pos - (double)i;
  return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

bool all_finite(const double* p, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

}  // namespace

extern "C" {

int tci_server_create(const tci_server_config* cfg, tci_server** out) {
  if (!cfg || !out) return TCI_ERR_ARG;
  *out = nullptr;
  if (cfg->slots < 1 || cfg->slots > 64 || cfg->planners < 1 || cfg->planners > 64 || cfg->hbm_budget_bytes <= 0 ||
      cfg->precision < 0 || cfg->precision > 1 || cfg->device < 0 || cfg->schedule_only_ms < 0 ||
      cfg->tc_gemms < 0 || cfg->tc_gemms > 2) {
    set_error("tci_server_create: slots and planners in 1..64, a positive budget, a known precision");
    return TCI_ERR_ARG;
  }
  try {
    std::unique_ptr<tci_server> s(new tci_server());
    s->cfg = *cfg;
    s->t0 = Clock::now();
    s->slot_req.resize(cfg->slots);
    s->slot_dead.assign(cfg->slots, 0);
    for (int64_t i = 0; i < cfg->planners; ++i) s->planners.emplace_back([p = s.get()] { p->planner_loop(); });
    for (int64_t i = 0; i < cfg->slots; ++i) s->workers.emplace_back([p = s.get(), i] { p->worker_loop((int)i); });
    s->supervisor = std::thread([p = s.get()] { p->supervisor_loop(); });
    *out = s.release();
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_server_submit(tci_server* s, const tci_deck* deck, const tci_operator* op, int64_t nroots, double tol_residual,
                      double tol_energy, int64_t maxit, int64_t* id) {
  if (!s || !deck || !op || !id || nroots <= 0) return TCI_ERR_ARG;
  try {
    auto r = std::make_shared<Request>();
    // copy the deck (and the arrays it points to) and the operator
    const int64_t nint = deck->num_inactive + deck->num_active;
    if (deck->num_orbitals <= 0 || nint <= 0 || nint >= deck->num_orbitals || deck->num_ref <= 0 || !deck->ref_occ)
      throw Error(TCI_ERR_INPUT, "inconsistent deck");
    r->deck = *deck;
    r->ref_occ.assign(deck->ref_occ, deck->ref_occ + deck->num_ref * nint);
    r->deck.ref_occ = r->ref_occ.data();
    if (deck->nm1_domain_ptr || deck->nm2_domain_ptr)
      throw Error(TCI_ERR_INPUT, "the server takes non-local decks (no pair domains)");
    if (!op->h || !op->chol || op->nchol <= 0) throw Error(TCI_ERR_ARG, "operator arrays are null");
    const size_t no = (size_t)deck->num_orbitals;
    const size_t nh = no * no, nl = no * (no + 1) / 2 * (size_t)op->nchol;
    // corrupted input is caught on the host before it reaches the device
    if (!all_finite(op->h, nh) || !all_finite(op->chol, nl) || !std::isfinite(op->core_energy))
      throw Error(TCI_ERR_INPUT, "operator holds non-finite values");
    if (!std::isfinite(tol_residual) || !std::isfinite(tol_energy)) throw Error(TCI_ERR_ARG, "non-finite tolerance");
    r->h.assign(op->h, op->h + nh);
    r->chol.assign(op->chol, op->chol + nl);
    r->nchol = op->nchol;
    r->core_energy = op->core_energy;
    r->nroots = nroots;
    r->maxit = maxit;
    r->tol_r = tol_residual;
    r->tol_e = tol_energy;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) throw Error(TCI_ERR_ARG, "server is shutting down");
    r->id = s->next_id++;
    r->t_submit = s->now();
    if (s->first_submit < 0) s->first_submit = r->t_submit;
    s->reqs[r->id] = r;
    s->to_plan.push_back(r);
    s->cv.notify_all();
    *id = r->id;
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_server_wait(tci_server* s, int64_t id, double timeout_s, double* energies, int64_t len, double* info) {
  if (!s) return TCI_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) {
    set_error("unknown request id");
    return TCI_ERR_ARG;
  }
  std::shared_ptr<Request> r = it->second;
  auto done = [&] { return r->state == RQ_DONE; };
  if (timeout_s < 0) {
    s->cv.wait(lk, done);
  } else if (!s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
    set_error("request not finished within the timeout");
    return TCI_ERR_TIMEOUT;
  }
  for (int64_t q = 0; energies && q < len && q < (int64_t)r->energies.size(); ++q) energies[q] = r->energies[q];
  if (info) {
    const double v[9] = {(double)r->status, (double)r->iterations, r->t_submit, r->t_planned, r->t_admitted,
                         r->t_done, r->est_bytes, (double)r->total_csfs, r->core_energy};
    std::memcpy(info, v, sizeof(v));
  }
  if (r->status != TCI_OK) set_error(r->error.empty() ? "request failed" : r->error);
  return r->status;
}

int tci_server_cancel(tci_server* s, int64_t id) {
  if (!s) return TCI_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) {
    set_error("unknown request id");
    return TCI_ERR_ARG;
  }
  std::shared_ptr<Request> r = it->second;
  if (r->state == RQ_DONE) return TCI_OK;
  if (r->state == RQ_RUNNING) {
    __atomic_store_n(&r->cancel, 1, __ATOMIC_RELEASE);
    return TCI_OK;
  }
  auto drop = [&](std::deque<std::shared_ptr<Request>>& q) { q.erase(std::remove(q.begin(), q.end(), r), q.end()); };
  drop(s->to_plan);
  drop(s->ready);
  s->finish(r, TCI_ERR_CANCELLED, "cancelled before it ran");
  return TCI_OK;
}

int tci_server_stats(tci_server* s, double* out, int64_t len) {
  if (!s || !out || len < 13) return TCI_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  const double span = s->last_done - s->first_submit;
  const double v[13] = {(double)s->reqs.size(),
                        (double)s->n_ok,
                        (double)s->n_failed,
                        (double)s->n_cancelled,
                        (double)(s->to_plan.size() + s->ready.size()),
                        (double)s->running,
                        (double)s->peak_running,
                        s->peak_reserved,
                        percentile(s->tts, 0.50),
                        percentile(s->tts, 0.99),
                        (s->n_ok > 0 && span > 0) ? (double)s->n_ok / span : 0.0,
                        (double)s->worker_restarts,
                        s->reserved};
  std::memcpy(out, v, sizeof(v));
  return TCI_OK;
}

void tci_server_destroy(tci_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    for (auto& kv : s->reqs)
      if (kv.second->state == RQ_RUNNING) __atomic_store_n(&kv.second->cancel, 1, __ATOMIC_RELEASE);
    s->cv.notify_all();
  }
  if (s->supervisor.joinable()) s->supervisor.join();
  for (auto& t : s->workers)
    if (t.joinable()) t.join();
  for (auto& t : s->planners)
    if (t.joinable()) t.join();
  delete s;
}

}  // extern "C"
