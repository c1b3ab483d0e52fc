// Denoising service: independent requests (one sample each) submitted at any
// time, batched on one device by length class and admitted by an estimate of
// their device-memory footprint; each batch runs through dgpu_dada_batch, so a
// request's result is exactly dgpu_dada's on that sample. The error model and
// the parameters are fixed for the service's lifetime. A request's input
// buffers are the caller's and must stay valid until its wait returns.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "dada2_b200.h"
#include "dgpu_common.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id = 0;
  int cls = 0;
  uint32_t n = 0;
  const char* seqs = nullptr;
  const uint32_t *offs = nullptr, *lens = nullptr, *abund = nullptr, *qsums = nullptr;
  const uint8_t* prior = nullptr;
  uint64_t total = 0, footprint = 0;
  Clock::time_point t_submit;
  dgpu_result* result = nullptr;
  int rc = 0;
  std::string err;
  double latency = 0.0;
  bool done = false;
};

// Length class of a request: its longest unique <= 200, <= 600 or longer.
// Uniques of one class share the aligner geometry of a batch.
int length_class(uint32_t lmax) { return lmax <= 200 ? 0 : (lmax <= 600 ? 1 : 2); }

// Concurrent batches: DGPU_SERVICE_WORKERS (1..16) if set, else 3.
int service_workers() {
  if (const char* e = std::getenv("DGPU_SERVICE_WORKERS")) {
    const int v = std::atoi(e);
    if (v >= 1 && v <= 16) return v;
  }
  return 3;
}

}  // namespace

namespace dgpu {
int dada_batch_each(int device, const dgpu_dada_params* params, int nsamples, const uint32_t* sample_start,
                    const char* seqs, const uint32_t* offs, const uint32_t* lens, const uint32_t* abund,
                    const uint8_t* prior, const uint32_t* qual_sums, const double* err_mat, int ncol,
                    const std::function<void(size_t, dgpu_result*)>& on_done);
}

// Requests wait in arrival order. Each worker takes the oldest pending
// request's length class and every pending request of that class in arrival
// order while the device-memory footprint of all batches in flight stays
// within the budget (a request is always admitted when nothing is in flight),
// and runs them as one batch; each request completes as soon as its own
// sample does. Several workers keep several batches on the device at once.
struct dgpu_service {
  int device = 0;
  dgpu_dada_params params{};
  std::vector<double> err;
  int ncol = 0;
  uint64_t budget = 0, in_flight = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::unordered_map<uint64_t, Request*> tickets;
  uint64_t next_id = 1;
  bool stop = false, held = false;
  uint64_t batches = 0, served = 0;
  std::vector<std::thread> workers;

  // under mu: the next batch if one is admissible now
  bool take(std::vector<Request*>& batch, uint64_t& used) {
    if (held || pending.empty()) return false;
    Request* first = pending.front();
    if (in_flight > 0 && in_flight + first->footprint > budget) return false;
    const int cls = first->cls;
    used = 0;
    for (auto it = pending.begin(); it != pending.end();) {
      Request* r = *it;
      if (r->cls == cls && (batch.empty() || in_flight + used + r->footprint <= budget)) {
        used += r->footprint;
        batch.push_back(r);
        it = pending.erase(it);
      } else {
        ++it;
      }
    }
    in_flight += used;
    return true;
  }

  void complete(Request* r) {  // under mu
    r->latency = std::chrono::duration<double>(Clock::now() - r->t_submit).count();
    r->done = true;
    served += 1;
    cv_done.notify_all();
  }

  void run() {
    if (cudaSetDevice(device) != cudaSuccess) {
      std::lock_guard<std::mutex> g(mu);
      stop = true;
      for (Request* r : pending) {
        r->rc = DGPU_E_CUDA;
        r->err = "cudaSetDevice failed in the service worker";
        complete(r);
      }
      pending.clear();
      cv_work.notify_all();
      return;
    }
    for (;;) {
      std::vector<Request*> batch;
      uint64_t used = 0;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return (stop && pending.empty()) || take(batch, used); });
        if (batch.empty()) return;  // stop requested and nothing left
        batches += 1;  // counted when taken: every batch is, before its requests complete
      }
      serve(batch);
      std::lock_guard<std::mutex> g(mu);
      in_flight -= used;
      cv_work.notify_all();
    }
  }

  void serve(std::vector<Request*>& batch) {
    const bool has_q = batch.front()->qsums != nullptr;
    bool same_q = true, any_prior = false;
    uint64_t total = 0;
    for (Request* r : batch) {
      same_q = same_q && (r->qsums != nullptr) == has_q;
      any_prior = any_prior || r->prior != nullptr;
      total += r->total;
    }
    std::vector<uint8_t> given(batch.size(), 0);
    if (batch.size() > 1 && same_q && total < 0xffffffffull) {
      // the batch's uniques packed back to back, request after request
      std::vector<uint32_t> start{0}, offs, lens, abund, qsums;
      std::vector<uint8_t> prior;
      std::vector<char> seqs(total);
      if (has_q) qsums.resize(total);
      uint64_t w = 0;
      for (Request* r : batch) {
        for (uint32_t t = 0; t < r->n; ++t) {
          offs.push_back(uint32_t(w));
          std::memcpy(seqs.data() + w, r->seqs + r->offs[t], r->lens[t]);
          if (has_q) std::memcpy(qsums.data() + w, r->qsums + r->offs[t], size_t(r->lens[t]) * 4);
          w += r->lens[t];
        }
        lens.insert(lens.end(), r->lens, r->lens + r->n);
        abund.insert(abund.end(), r->abund, r->abund + r->n);
        if (any_prior) {
          if (r->prior) prior.insert(prior.end(), r->prior, r->prior + r->n);
          else prior.insert(prior.end(), r->n, 0);
        }
        start.push_back(start.back() + r->n);
      }
      dgpu::dada_batch_each(device, &params, int(batch.size()), start.data(), seqs.data(), offs.data(), lens.data(),
                            abund.data(), any_prior ? prior.data() : nullptr, has_q ? qsums.data() : nullptr,
                            err.data(), ncol, [&](size_t i, dgpu_result* res) {
                              std::lock_guard<std::mutex> g(mu);
                              batch[i]->result = res;
                              given[i] = 1;
                              complete(batch[i]);
                            });
      // a request with invalid input (or a device failure) fails the batch:
      // what was not handed over is served alone, so each gets its own outcome
    }
    for (size_t i = 0; i < batch.size(); ++i) {
      if (given[i]) continue;
      Request* r = batch[i];
      dgpu_result* res = nullptr;
      const int rc = dgpu_dada(device, &params, int(r->n), r->seqs, r->offs, r->lens, r->abund, r->prior, r->qsums,
                               err.data(), ncol, &res);
      std::lock_guard<std::mutex> g(mu);
      r->rc = rc;
      if (rc) r->err = dgpu_last_error();
      r->result = res;
      complete(r);
    }
  }
};

extern "C" {

int dgpu_service_create(int device, const dgpu_dada_params* params, const double* err_mat, int ncol,
                        uint64_t hbm_budget, dgpu_service** out) {
  if (!params || !err_mat || ncol <= 0 || !out) {
    dgpu::set_last_error("null argument or ncol <= 0");
    return DGPU_E_INVALID;
  }
  uint64_t budget = hbm_budget;
  if (budget == 0) {
    int prev = 0;
    cudaGetDevice(&prev);
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      dgpu::set_last_error("cannot query the device's memory");
      return DGPU_E_CUDA;
    }
    cudaSetDevice(prev);
    budget = uint64_t(free_b) / 2;
  }
  dgpu_service* s = new dgpu_service();
  s->device = device;
  s->params = *params;
  s->err.assign(err_mat, err_mat + 16 * size_t(ncol));
  s->ncol = ncol;
  s->budget = budget;
  const int nw = service_workers();
  for (int k = 0; k < nw; ++k) s->workers.emplace_back([s] { s->run(); });
  *out = s;
  return 0;
}

int dgpu_service_submit(dgpu_service* s, int nraw, const char* seqs, const uint32_t* offs, const uint32_t* lens,
                        const uint32_t* abund, const uint8_t* prior, const uint32_t* qual_sums, uint64_t* ticket) {
  if (!s || nraw <= 0 || !seqs || !offs || !lens || !abund || !ticket) {
    dgpu::set_last_error("null argument or no uniques");
    return DGPU_E_INVALID;
  }
  Request* r = new Request();
  r->t_submit = Clock::now();
  r->n = uint32_t(nraw);
  r->seqs = seqs;
  r->offs = offs;
  r->lens = lens;
  r->abund = abund;
  r->prior = prior;
  r->qsums = qual_sums;
  uint32_t lmax = 0;
  for (int t = 0; t < nraw; ++t) {
    r->total += lens[t];
    lmax = std::max(lmax, lens[t]);
  }
  const uint64_t total = r->total;
  r->cls = length_class(lmax);
  // device bytes while served: codes and qualities, the k-mer screen, per-raw
  // state, and the aligners' per-warp pointer scratch of its batch
  const int k = s->params.align.kmer_size;
  const uint64_t profile = k >= 8 ? 3 * uint64_t(lmax) : (uint64_t(1) << (2 * k));
  r->footprint = 2 * total + uint64_t(r->n) * (profile + 64) + uint64_t(2 * lmax + 1) * 32 * 2368 * 3;
  std::lock_guard<std::mutex> g(s->mu);
  if (s->stop) {
    delete r;
    dgpu::set_last_error("service stopped");
    return DGPU_E_INVALID;
  }
  r->id = s->next_id++;
  s->tickets[r->id] = r;
  s->pending.push_back(r);
  *ticket = r->id;
  s->cv_work.notify_one();
  return 0;
}

int dgpu_service_wait(dgpu_service* s, uint64_t ticket, dgpu_result** out, double* latency_s) {
  if (!s || !out) {
    dgpu::set_last_error("null argument");
    return DGPU_E_INVALID;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) {
    dgpu::set_last_error("unknown ticket");
    return DGPU_E_INVALID;
  }
  Request* r = it->second;
  s->cv_done.wait(lk, [&] { return r->done; });
  s->tickets.erase(it);
  lk.unlock();
  const int rc = r->rc;
  if (latency_s) *latency_s = r->latency;
  if (rc) dgpu::set_last_error(r->err.c_str());
  *out = r->result;
  delete r;
  return rc;
}

int dgpu_service_stats(dgpu_service* s, uint64_t* batches, uint64_t* served) {
  if (!s) {
    dgpu::set_last_error("null argument");
    return DGPU_E_INVALID;
  }
  std::lock_guard<std::mutex> g(s->mu);
  if (batches) *batches = s->batches;
  if (served) *served = s->served;
  return 0;
}

int dgpu_service_hold(dgpu_service* s, int hold) {
  if (!s) {
    dgpu::set_last_error("null argument");
    return DGPU_E_INVALID;
  }
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->held = hold != 0;
  }
  s->cv_work.notify_all();
  return 0;
}

void dgpu_service_destroy(dgpu_service* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    s->held = false;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();  // serves what was already submitted
  for (auto& kv : s->tickets) {
    if (kv.second->result) dgpu_result_free(kv.second->result);
    delete kv.second;
  }
  delete s;
}

}  // extern "C"
