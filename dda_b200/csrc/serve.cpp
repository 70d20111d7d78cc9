// serve.cpp -- the request loop of include/dda_serve.h.
//
// Worker threads (one per slot) take queued requests in arrival order; a
// request is admitted when its footprint fits the unused budget.  A later,
// smaller request may go ahead of the head of the queue while the head does
// not fit, at most kMaxBypass times, after which the head is waited for.
// Each admitted request runs on its own context and stream: geometry and
// incident fields from the front end, dda_create (D-matrix on the GPU),
// dda_solve, the forward far field for the cross sections, dda_destroy.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dda_cuda.h"
#include "../../include/dda_frontend.h"
#include "../../include/dda_serve.h"

namespace {

thread_local std::string g_serve_err;
constexpr int kMaxBypass = 8;

struct Job {
  int64_t id = 0;
  dda_serve_request req{};
  std::vector<uint32_t> pos;
  std::vector<uint8_t> mat;
  std::vector<double> refr;
  std::string grid_unit, wavelength;
  dda_problem prob{};
  int64_t peak = 0;
  double t_submit = 0;
  int bypassed = 0;
};

struct Done {
  dda_serve_result res{};
  std::vector<double> pol;
};

}  // namespace

struct dda_server {
  int device = 0;
  int64_t budget = 0;
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::unique_ptr<Job>> queue;
  std::deque<std::unique_ptr<Done>> done;
  std::map<int64_t, std::unique_ptr<Done>> held;  // results with kept polarisations
  std::map<int64_t, dda_ctx*> active;             // running requests' contexts (dda_serve_cancel)
  std::set<int64_t> running_ids;                  // admitted, not finished
  std::set<int64_t> cancel_asked;                 // running requests cancelled before their context existed
  int64_t used = 0;
  int64_t running = 0;
  int64_t next_id = 1;
  bool stopping = false;
  std::vector<std::thread> workers;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  void worker();
  void run(Job& j, Done& d);
};

namespace {

void set_error(Done& d, const std::string& msg, int code) {
  d.res.status = code;
  std::snprintf(d.res.error, sizeof(d.res.error), "%s", msg.c_str());
}

}  // namespace

// One request: the sequence of ddaMain for one target (DDA/DDAMain.cpp:611-771).
void dda_server::run(Job& j, Done& d) {
  nvtxRangePushA("dda served request");
  struct Pop {
    ~Pop() { nvtxRangePop(); }
  } pop;
  const dda_serve_request& q = j.req;
  d.res.npol = q.npol;
  if (cudaSetDevice(device) != cudaSuccess) return set_error(d, "cudaSetDevice failed", DDA_ERR_CUDA);
  dda_geometry* g = nullptr;
  if (dda_geom_from_arrays(j.pos.data(), j.mat.empty() ? nullptr : j.mat.data(), q.nv, j.grid_unit.c_str(), &g))
    return set_error(d, dda_frontend_error(), DDA_ERR_ARG);
  std::unique_ptr<dda_geometry, void (*)(dda_geometry*)> gg(g, dda_geom_free);
  double lambda = 0;
  if (dda_parse_length_m(j.wavelength.c_str(), &lambda) || !(lambda > 0))
    return set_error(d, "bad wavelength", DDA_ERR_ARG);
  const double d_m = dda_geom_grid_unit(g);
  const double k = 2 * M_PI / lambda;
  dda_problem P = j.prob;
  P.positions = dda_geom_positions(g);
  P.materials = dda_geom_materials(g);
  P.kd = k * d_m;
  P.grid_unit = d_m;
  dda_ctx* ctx = nullptr;
  int rc = dda_create(&P, q.precision, &ctx);
  if (rc != DDA_OK) return set_error(d, dda_last_error(nullptr), rc);
  std::unique_ptr<dda_ctx, int (*)(dda_ctx*)> cc(ctx, dda_destroy);
  // registered for dda_serve_cancel while it exists (unregistered before
  // the context is destroyed: `reg` is released before `cc`)
  {
    std::lock_guard<std::mutex> lk(mu);
    active[j.id] = ctx;
    if (cancel_asked.erase(j.id)) dda_cancel(ctx);
  }
  auto unreg = [this, &j](void*) {
    std::lock_guard<std::mutex> lk(mu);
    active.erase(j.id);
  };
  std::unique_ptr<void, decltype(unreg)> reg(ctx, unreg);
  d.res.t_setup = now();
  int64_t layout[8] = {};
  dda_matvec_layout(ctx, layout);
  d.res.device_bytes = layout[7];
  const int64_t nvs = dda_vec_stride(ctx);
  d.res.nvs = nvs;
  const size_t vlen = (size_t)3 * nvs * 2;  // doubles per right-hand side
  const int pol0 = (q.npol == 1 && q.first_pol == 2) ? 2 : 1;  // polarisation of right-hand side 0
  std::vector<double> einc(vlen * q.npol), cc_all(q.nmat * 6 * q.npol);
  for (int r = 0; r < q.npol; r++) {
    std::vector<double> ccv(q.nmat * 6), ccs(q.nmat * 6), chi(q.nmat * 6);
    if (dda_couple_constants(q.polarizability, q.nmat, j.refr.data(), d_m, k, q.prop, pol0 + r, ccv.data(),
                             ccs.data(), chi.data()))
      return set_error(d, dda_frontend_error(), DDA_ERR_ARG);
    std::copy(ccv.begin(), ccv.end(), cc_all.begin() + (size_t)r * q.nmat * 6);
    if ((rc = dda_set_cc(ctx, r, ccs.data())) != DDA_OK) return set_error(d, dda_last_error(ctx), rc);
    if (dda_einc_plane(g, k, q.prop, pol0 + r, einc.data() + r * vlen))
      return set_error(d, dda_frontend_error(), DDA_ERR_ARG);
  }
  d.pol.assign(vlen * q.npol, 0.0);
  rc = dda_solve(ctx, q.solver, q.npol, einc.data(), q.eps, q.max_iter, nullptr, d.pol.data(), nullptr, 0,
                 d.res.stats);
  d.res.t_solved = now();
  if (rc != DDA_OK) {
    set_error(d, dda_last_error(ctx), rc);
    if (!q.keep_pol) d.pol.clear();
    return;
  }
  // cross sections: far field in the propagation direction (PlaneWave::extCross,
  // DDA/Beam.cpp:126-133) and the absorbed power (AbsCross::absCross,
  // DDA/AbsCross.cpp:28-48)
  double inc[3], pn[3];
  dda_beam_pol(q.prop, 1, inc, pn);
  std::vector<double> ef((size_t)q.npol * 6);
  if ((rc = dda_far_field(ctx, q.npol, nullptr, 1, pn, ef.data())) != DDA_OK)
    return set_error(d, dda_last_error(ctx), rc);
  const double four_pi = 4 * M_PI, temp1 = k * k * k * 2 / 3;
  for (int r = 0; r < q.npol; r++) {
    dda_beam_pol(q.prop, pol0 + r, inc, pn);
    const double* e = ef.data() + (size_t)r * 6;
    d.res.cext[r] = -(e[0] * inc[0] + e[2] * inc[1] + e[4] * inc[2]) * four_pi / k;
    const std::complex<double>* ccr = reinterpret_cast<const std::complex<double>*>(cc_all.data()) + (size_t)r * q.nmat * 3;
    const double* pr = d.pol.data() + r * vlen;
    const uint8_t* mat = dda_geom_materials(g);
    double sum = 0;
    for (int c = 0; c < 3; c++) {
      std::vector<double> mdr(q.nmat);
      for (uint32_t m = 0; m < q.nmat; m++) mdr[m] = -std::imag(1.0 / ccr[m * 3 + c]) - temp1;
      for (uint32_t i = 0; i < q.nv; i++) {
        const double re = pr[2 * (i + (size_t)c * nvs)], im = pr[2 * (i + (size_t)c * nvs) + 1];
        sum += mdr[mat[i]] * (re * re + im * im);
      }
    }
    d.res.cabs[r] = four_pi * k * sum;
  }
  if (!q.keep_pol) d.pol.clear();
}

void dda_server::worker() {
  for (;;) {
    std::unique_ptr<Job> job;
    {
      std::unique_lock<std::mutex> lk(mu);
      for (;;) {
        if (queue.empty()) {
          if (stopping) return;
          cv_work.wait(lk);
          continue;
        }
        auto it = queue.end();
        if (used + queue.front()->peak <= budget) {
          it = queue.begin();
        } else if (queue.front()->bypassed < kMaxBypass) {
          it = std::find_if(queue.begin() + 1, queue.end(),
                            [&](const std::unique_ptr<Job>& j) { return used + j->peak <= budget; });
          if (it != queue.end()) queue.front()->bypassed++;
        }
        if (it != queue.end()) {
          job = std::move(*it);
          queue.erase(it);
          break;
        }
        cv_work.wait(lk);  // a finishing request frees budget
      }
      used += job->peak;
      running++;
      running_ids.insert(job->id);
    }
    std::unique_ptr<Done> d(new Done);
    d->res.id = job->id;
    d->res.tag = job->req.tag;
    d->res.t_submit = job->t_submit;
    d->res.t_admit = now();
    d->res.footprint = job->peak;
    d->res.nv = job->req.nv;
    for (int a = 0; a < 3; a++) d->res.grid[a] = job->prob.grid[a];
    try {
      run(*job, *d);
    } catch (const std::exception& e) {
      set_error(*d, e.what(), DDA_ERR_ARG);
    }
    d->res.t_done = now();
    {
      std::lock_guard<std::mutex> lk(mu);
      used -= job->peak;
      running--;
      running_ids.erase(job->id);
      cancel_asked.erase(job->id);
      done.push_back(std::move(d));
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
}

extern "C" {

const char* dda_serve_error(void) { return g_serve_err.c_str(); }

int dda_serve_create(int device, int64_t hbm_budget, int max_active, dda_server** out) {
  if (!out || max_active < 1) {
    g_serve_err = "bad arguments";
    return DDA_ERR_ARG;
  }
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    g_serve_err = "cudaSetDevice failed";
    return DDA_ERR_CUDA;
  }
  if (hbm_budget <= 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      g_serve_err = "cudaMemGetInfo failed";
      return DDA_ERR_CUDA;
    }
    hbm_budget = (int64_t)(0.9 * (double)fr);
  }
  // Contexts allocate from the device's default memory pool on their
  // streams.  Let the pool keep up to the budget mapped between requests
  // instead of returning memory to the driver at every synchronisation
  // (a process-local pool attribute).
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = (uint64_t)hbm_budget;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  dda_server* s = new dda_server;
  s->device = device;
  s->budget = hbm_budget;
  s->t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < max_active; i++) s->workers.emplace_back([s] { s->worker(); });
  *out = s;
  return DDA_OK;
}

int dda_serve_submit(dda_server* s, const dda_serve_request* q, int64_t* id) {
  if (!s || !q || !q->positions || q->nv == 0 || q->nmat == 0 || q->nmat > 256 || !q->refr || !q->grid_unit ||
      !q->wavelength || q->npol < 1 || q->npol > 2) {
    g_serve_err = "bad request";
    return DDA_ERR_ARG;
  }
  std::unique_ptr<Job> j(new Job);
  j->req = *q;
  j->pos.assign(q->positions, q->positions + (size_t)q->nv * 3);
  if (q->materials) j->mat.assign(q->materials, q->materials + q->nv);
  j->refr.assign(q->refr, q->refr + (size_t)q->nmat * 6);
  j->grid_unit = q->grid_unit;
  j->wavelength = q->wavelength;
  j->req.positions = nullptr;
  j->req.materials = nullptr;
  j->req.refr = nullptr;
  j->req.grid_unit = nullptr;
  j->req.wavelength = nullptr;
  // box and grid as DDAParams chooses them (DDA/DDAParams.cpp:290-335)
  uint32_t box[3] = {0, 0, 0};
  for (uint32_t i = 0; i < q->nv; i++)
    for (int a = 0; a < 3; a++) box[a] = std::max(box[a], j->pos[3 * i + a] + 1);
  dda_problem& P = j->prob;
  P.nv = q->nv;
  P.nmat = q->nmat;
  P.max_rhs = q->npol;
  P.device = s->device;
  for (int a = 0; a < 3; a++) P.box[a] = box[a];
  if (dda_choose_grid(box, q->grid_policy, P.grid) != DDA_OK) {
    g_serve_err = "bad grid policy";
    return DDA_ERR_ARG;
  }
  int64_t resident = 0;
  if (dda_footprint(&P, q->precision, &resident, &j->peak) != DDA_OK) {
    g_serve_err = "bad precision";
    return DDA_ERR_ARG;
  }
  if (j->peak > s->budget) {
    g_serve_err = "request footprint " + std::to_string(j->peak) + " bytes exceeds the budget of " +
                  std::to_string(s->budget);
    return DDA_ERR_OOM;
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) {
      g_serve_err = "server is stopping";
      return DDA_ERR_ARG;
    }
    j->id = s->next_id++;
    j->t_submit = s->now();
    if (id) *id = j->id;
    s->queue.push_back(std::move(j));
  }
  s->cv_work.notify_all();
  return DDA_OK;
}

int dda_serve_poll(dda_server* s, dda_serve_result* out, int max, int timeout_ms) {
  if (!s || !out || max < 1) return DDA_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto ready = [&] { return !s->done.empty(); };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, [&] { return ready() || (s->queue.empty() && s->running == 0); });
  } else if (timeout_ms > 0) {
    s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
  }
  int n = 0;
  while (n < max && !s->done.empty()) {
    std::unique_ptr<Done> d = std::move(s->done.front());
    s->done.pop_front();
    out[n] = d->res;
    out[n].pol = d->pol.empty() ? nullptr : d->pol.data();
    if (!d->pol.empty()) s->held[d->res.id] = std::move(d);
    n++;
  }
  return n;
}

int dda_serve_cancel(dda_server* s, int64_t id) {
  if (!s) return DDA_ERR_ARG;
  std::unique_ptr<Done> d;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = std::find_if(s->queue.begin(), s->queue.end(),
                           [&](const std::unique_ptr<Job>& j) { return j->id == id; });
    if (it != s->queue.end()) {  // still queued: never admitted
      d.reset(new Done);
      d->res.id = id;
      d->res.tag = (*it)->req.tag;
      d->res.npol = (*it)->req.npol;
      d->res.nv = (*it)->req.nv;
      d->res.t_submit = (*it)->t_submit;
      d->res.t_admit = d->res.t_done = s->now();
      for (int a = 0; a < 3; a++) d->res.grid[a] = (*it)->prob.grid[a];
      set_error(*d, "cancelled before admission", DDA_ERR_CANCELLED);
      s->queue.erase(it);
      s->done.push_back(std::move(d));
    } else {
      auto a = s->active.find(id);
      if (a != s->active.end()) {
        dda_cancel(a->second);  // the solve stops after its current round
      } else if (s->running_ids.count(id)) {
        s->cancel_asked.insert(id);  // admitted, context not built yet
      } else {
        return DDA_ERR_ARG;
      }
      return DDA_OK;
    }
  }
  s->cv_done.notify_all();
  s->cv_work.notify_all();
  return DDA_OK;
}

int dda_serve_release(dda_server* s, int64_t id) {
  if (!s) return DDA_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->held.erase(id);
  return DDA_OK;
}

int64_t dda_serve_pending(dda_server* s) {
  if (!s) return 0;
  std::lock_guard<std::mutex> lk(s->mu);
  return (int64_t)s->queue.size() + s->running;
}

double dda_serve_clock(const dda_server* s) { return s ? s->now() : 0.0; }

int dda_serve_destroy(dda_server* s) {
  if (!s) return DDA_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  delete s;
  return DDA_OK;
}

}  // extern "C"
