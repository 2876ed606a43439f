// Serving loop: continuous batching of SIMP jobs on one GPU (no counterpart in the reference, whose App runs
// one optimisation at a time through the FemWorkTeam lock, src/Mycel.Core/Fem/FemWorkTeam.cs:109).
//
// A server owns `slots` worker threads, each with its own mycel_ctx (CUDA stream). A worker takes the next
// admissible job, keeps its state resident on the device for all its SIMP iterations (mycel_simp_begin /
// step / read / end on a problem of its own), and releases the job's device memory when it ends. Kernels of
// different jobs run concurrently on their streams, so the PCG iterations of the running jobs interleave on
// the device. Admission is in arrival order, with backfill: when the oldest queued job does not fit in what
// is left of the HBM budget, a later job that fits may start first. A job larger than the whole budget fails
// with MYCEL_E_OOM. Device allocation is stream-ordered (cudaMallocAsync), so one job's set-up and tear-down
// do not synchronise the device under the others.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  int64_t id = 0;
  mycel_grid grid{};
  std::vector<uint8_t> domain;
  mycel_material material{};
  std::vector<int32_t> fixed;
  std::vector<std::vector<int32_t>> load_nodes;
  std::vector<std::vector<double>> load_area;
  std::vector<mycel_load_case> loads;
  std::vector<double> density;
  double penal = 3.0;
  mycel_simp_options opt{};
  std::vector<uint8_t> passive;
  std::vector<float> init_density;
  std::vector<double> warm;
  int keep_u = 0;
  int64_t bytes = 0;
  // state and results (guarded by the server mutex once the job is shared)
  int state = MYCEL_JOB_QUEUED;
  int32_t status = MYCEL_OK;
  std::string message;
  double t_submit = 0, t_start = 0, t_finish = 0;
  int iterations = 0, converged = 0;
  int64_t solver_iterations = 0;
  double final_compliance = 0;
  std::vector<mycel_iter_record> history;
  std::vector<float> phys, des;
  std::vector<double> u;
};

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  // nearest-rank percentile
  size_t k = (size_t)std::ceil(q * (double)v.size());
  if (k < 1) k = 1;
  if (k > v.size()) k = v.size();
  return v[k - 1];
}

int64_t al16(int64_t b) { return (std::max<int64_t>(b, 16) + 15) & ~int64_t(15); }

}  // namespace

struct mycel_server {
  mycel_server_options opt{};
  Clock::time_point t0;
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  std::deque<Job*> queue;
  std::map<int64_t, std::unique_ptr<Job>> jobs;
  int64_t next_id = 0;
  int64_t admitted = 0, peak = 0;
  int running = 0;
  bool stopping = false;
  std::vector<mycel_ctx*> ctxs;
  std::vector<std::thread> workers;
  std::string last_error;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  void worker(int slot);
  void run(Job* j, mycel_ctx* c);
};

// Device memory of one job, allocation by allocation as problem_create, ensure_pcg_workspace, ensure_mixed,
// filter_create and simp_begin make them (each rounded to 16 bytes as they count it).
static int64_t job_bytes(const mycel_grid& gr, int64_t n_active, int64_t n_fixed, int64_t n_load_nodes,
                         int32_t n_loads, const mycel_simp_options& o, int num_sms) {
  const mycel::GridDims g = mycel::make_dims(gr.nx, gr.ny, gr.nz);
  const int64_t ne = g.ne, nn = g.nn, nd = g.nd, na = std::max<int64_t>(n_active, 1);
  const int64_t nfnz = std::max<int64_t>(std::min<int64_t>(3 * n_load_nodes, nd), 1);
  int64_t b = 0;
  // problem
  b += al16(ne) + al16((nn + 3) & ~int64_t(3)) + al16(4 * na) + al16(8 * nd) + al16(8 * nd) + 2 * al16(4 * nfnz) +
       al16(8 * ne) + al16(8 * ne) + al16(4 * ne) + al16(8 * nd) + al16(8 * nd) + al16(4 * g.n32) + al16(8 * nd) +
       al16(8 * nd) + al16(4 * std::max<int64_t>(n_fixed, 1)) + al16(4) + al16(4) +
       al16(8 * std::max<int64_t>(nd / 256 + 1024, 65536));
  // PCG workspace
  const int64_t nb = (nd + 8191) / 8192;
  b += 5 * al16(8 * nd) + al16(8 * (2 * nb + 64)) + al16(sizeof(mycel::PcgState));
  // mixed workspace (6 FP32 vectors) and the fast FP64 workspace (7 FP64 vectors) a mixed solve escalates to
  const bool mg = o.precision == MYCEL_PRECISION_FP64_MG || o.precision == MYCEL_PRECISION_MIXED_MG;
  if (o.precision == MYCEL_PRECISION_MIXED || mg) b += 6 * (4 * g.n32 + 64);
  if (o.precision == MYCEL_PRECISION_MIXED || o.precision == MYCEL_PRECISION_FP64_FACTORED || mg)
    b += 7 * (8 * g.n64 + 64);
  if (mg)
    b += mycel::mg_device_bytes(g.nx, g.ny, g.nz, n_loads,
                                o.precision == MYCEL_PRECISION_MIXED_MG && o.separate_load_cases != 0);
  // filter (stencil offsets and weights of radius ceil(rmin) <= max(filter radius, 1.5) / h, plus invHs, S)
  double rmin = o.filter_radius_mm / std::max(1e-30, (double)gr.h);
  if (o.enforce_minimum_filter_radius && rmin < 1.5) rmin = 1.5;
  const int64_t r = (int64_t)std::ceil(rmin) + 1, n_off = (2 * r + 1) * (2 * r + 1) * (2 * r + 1);
  b += 16 * n_off + 8 * n_off + 16 * ne;
  // SIMP session
  b += 5 * al16(8 * ne) + al16(8 * nd) + al16(8 * 16) + al16(8 * ((int64_t)num_sms * 16 + 64)) +
       al16(sizeof(mycel::OcOut)) + al16(ne) + 2 * al16(4 * ne);
  if (o.enable_heaviside) b += 2 * al16(8 * ne);
  // load cases apart: F_k and P F_k, their non-zero lists, each case's u, the per-case compliances
  if (o.separate_load_cases && n_loads > 1)
    b += 3 * al16(8 * (int64_t)n_loads * nd) + al16(4 * std::max<int64_t>(6 * n_load_nodes, 1)) + al16(8 * n_loads);
  return b;
}

static int64_t spec_bytes(const mycel_job_spec* j, int num_sms) {
  const mycel::GridDims g = mycel::make_dims(j->grid.nx, j->grid.ny, j->grid.nz);
  int64_t na = 0;
  if (j->domain)
    for (int64_t e = 0; e < g.ne; ++e) na += j->domain[e] != 0;
  int64_t nl = 0;
  for (int32_t q = 0; q < j->n_loads; ++q) nl += j->loads[q].n_nodes;
  return job_bytes(j->grid, na, j->n_fixed, nl, j->n_loads, j->options, num_sms);
}

extern "C" int64_t mycel_job_device_bytes(const mycel_job_spec* job) {
  if (!job || job->grid.nx <= 0 || job->grid.ny <= 0 || job->grid.nz <= 0) return -1;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  (void)cudaGetLastError();
  return spec_bytes(job, sms);
}

void mycel_server::run(Job* j, mycel_ctx* c) {
  mycel_problem* p = nullptr;
  mycel_simp_session* ss = nullptr;
  int32_t rc = mycel_problem_create(c, &j->grid, j->domain.data(), &j->material, j->fixed.data(),
                                    (int32_t)j->fixed.size(), j->loads.data(), (int32_t)j->loads.size(),
                                    j->density.empty() ? nullptr : j->density.data(), j->penal, &p);
  if (!rc) rc = mycel_simp_begin(p, &j->opt, &ss);
  std::vector<mycel_iter_record> hist;
  int64_t solver = 0;
  int32_t done = 0;
  while (!rc && !done) {
    mycel_iter_record r;
    rc = mycel_simp_step(ss, &r, &done);
    if (!rc) {
      hist.push_back(r);
      solver += r.solver_iterations;
    }
  }
  std::vector<float> phys, des;
  std::vector<double> u;
  if (!rc) {
    phys.resize((size_t)((int64_t)j->grid.nx * j->grid.ny * j->grid.nz));
    des.resize(phys.size());
    if (j->keep_u) u.resize((size_t)(3 * (int64_t)(j->grid.nx + 1) * (j->grid.ny + 1) * (j->grid.nz + 1)));
    rc = mycel_simp_read(ss, j->keep_u ? u.data() : nullptr, phys.data(), des.data(), nullptr, nullptr, nullptr);
  }
  std::string msg = rc ? std::string(mycel_last_error(c)) : std::string();
  int conv = 0;
  if (ss) {
    conv = mycel::simp_session_converged(ss) ? 1 : 0;
    mycel_simp_end(ss);
  }
  if (p) mycel_problem_destroy(p);
  cudaStreamSynchronize(c->stream);  // the job's memory is back in the pool before its bytes are released
  std::lock_guard<std::mutex> lk(m);
  j->status = rc;
  j->message = msg;
  j->state = rc ? MYCEL_JOB_FAILED : MYCEL_JOB_DONE;
  j->iterations = (int)hist.size();
  j->converged = conv;
  j->solver_iterations = solver;
  j->final_compliance = hist.empty() ? 0.0 : hist.back().compliance;
  j->history = std::move(hist);
  j->phys = std::move(phys);
  j->des = std::move(des);
  j->u = std::move(u);
  j->t_finish = now();
}

void mycel_server::worker(int slot) {
  mycel_ctx* c = ctxs[(size_t)slot];
  cudaSetDevice(c->device);
  std::unique_lock<std::mutex> lk(m);
  for (;;) {
    Job* j = nullptr;
    cv_work.wait(lk, [&] {
      if (stopping) return true;
      for (Job* q : queue)
        if (admitted + q->bytes <= opt.hbm_budget_bytes) return true;
      return false;
    });
    if (stopping) return;
    for (auto it = queue.begin(); it != queue.end(); ++it)
      if (admitted + (*it)->bytes <= opt.hbm_budget_bytes) {
        j = *it;
        queue.erase(it);
        break;
      }
    if (!j) continue;
    admitted += j->bytes;
    peak = std::max(peak, admitted);
    ++running;
    j->state = MYCEL_JOB_RUNNING;
    j->t_start = now();
    lk.unlock();
    run(j, c);
    lk.lock();
    admitted -= j->bytes;
    --running;
    cv_done.notify_all();
    cv_work.notify_all();
  }
}

extern "C" int32_t mycel_server_create(const mycel_server_options* opt, mycel_server** out) {
  if (!opt || !out) return mycel::set_error(nullptr, MYCEL_E_ARG, "NULL argument");
  *out = nullptr;
  if (opt->slots < 1 || opt->hbm_budget_bytes <= 0) return mycel::set_error(nullptr, MYCEL_E_ARG, "slots and hbm_budget_bytes must be positive");
  auto* s = new mycel_server();
  s->opt = *opt;
  s->t0 = Clock::now();
  for (int q = 0; q < opt->slots; ++q) {
    mycel_ctx* c = nullptr;
    int32_t rc = mycel_ctx_create(opt->device, &c);
    if (rc) {
      for (mycel_ctx* x : s->ctxs) mycel_ctx_destroy(x);
      delete s;
      return rc;
    }
    s->ctxs.push_back(c);
  }
  for (int q = 0; q < opt->slots; ++q) s->workers.emplace_back(&mycel_server::worker, s, q);
  *out = s;
  return MYCEL_OK;
}

extern "C" int32_t mycel_server_submit(mycel_server* s, const mycel_job_spec* js, int64_t* job_id) {
  if (!s || !js || !job_id) return mycel::set_error(nullptr, MYCEL_E_ARG, "NULL argument");
  const mycel_grid& gr = js->grid;
  if (gr.nx <= 0 || gr.ny <= 0 || gr.nz <= 0 || !js->domain) {
    std::lock_guard<std::mutex> lk(s->m);
    s->last_error = "job grid must be positive and domain non-NULL";
    return MYCEL_E_ARG;
  }
  auto j = std::make_unique<Job>();
  const mycel::GridDims g = mycel::make_dims(gr.nx, gr.ny, gr.nz);
  j->grid = gr;
  j->domain.assign(js->domain, js->domain + g.ne);
  j->material = js->material;
  if (js->n_fixed > 0) j->fixed.assign(js->fixed_dofs, js->fixed_dofs + js->n_fixed);
  for (int32_t q = 0; q < js->n_loads; ++q) {
    const mycel_load_case& lc = js->loads[q];
    j->load_nodes.emplace_back(lc.nodes, lc.nodes + std::max(lc.n_nodes, 0));
    if (lc.node_area) j->load_area.emplace_back(lc.node_area, lc.node_area + std::max(lc.n_nodes, 0));
    else j->load_area.emplace_back();
  }
  for (int32_t q = 0; q < js->n_loads; ++q) {
    mycel_load_case lc = js->loads[q];
    lc.nodes = j->load_nodes[(size_t)q].data();
    lc.node_area = js->loads[q].node_area ? j->load_area[(size_t)q].data() : nullptr;
    j->loads.push_back(lc);
  }
  if (js->element_density) j->density.assign(js->element_density, js->element_density + g.ne);
  j->penal = js->penal;
  j->opt = js->options;
  if (js->options.passive_mask && js->options.passive_mask_len > 0) {
    j->passive.assign(js->options.passive_mask, js->options.passive_mask + js->options.passive_mask_len);
    j->opt.passive_mask = j->passive.data();
  }
  if (js->options.initial_density && js->options.initial_density_len > 0) {
    j->init_density.assign(js->options.initial_density, js->options.initial_density + js->options.initial_density_len);
    j->opt.initial_density = j->init_density.data();
  }
  if (js->options.warm_start_displacements && js->options.warm_start_len > 0) {
    j->warm.assign(js->options.warm_start_displacements, js->options.warm_start_displacements + js->options.warm_start_len);
    j->opt.warm_start_displacements = j->warm.data();
  }
  j->keep_u = js->keep_u;
  j->bytes = spec_bytes(js, s->ctxs.empty() ? 148 : s->ctxs[0]->num_sms);
  std::lock_guard<std::mutex> lk(s->m);
  j->id = s->next_id++;
  j->t_submit = s->now();
  *job_id = j->id;
  Job* raw = j.get();
  s->jobs[j->id] = std::move(j);
  if (raw->bytes > s->opt.hbm_budget_bytes) {
    raw->state = MYCEL_JOB_FAILED;
    raw->status = MYCEL_E_OOM;
    raw->message = "job needs " + std::to_string(raw->bytes) + " bytes of device memory, more than the server's budget";
    raw->t_start = raw->t_finish = raw->t_submit;
    s->cv_done.notify_all();
    return MYCEL_OK;
  }
  s->queue.push_back(raw);
  s->cv_work.notify_all();
  return MYCEL_OK;
}

extern "C" int32_t mycel_server_job_info(mycel_server* s, int64_t id, mycel_job_info* o) {
  if (!s || !o) return mycel::set_error(nullptr, MYCEL_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->m);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) {
    s->last_error = "unknown job id";
    return MYCEL_E_ARG;
  }
  const Job& j = *it->second;
  std::memset(o, 0, sizeof *o);
  o->state = j.state;
  o->status = j.status;
  o->iterations = j.iterations;
  o->converged = j.converged;
  o->device_bytes = j.bytes;
  o->submit_s = j.t_submit;
  o->start_s = j.t_start;
  o->finish_s = j.t_finish;
  o->final_compliance = j.final_compliance;
  o->solver_iterations = j.solver_iterations;
  std::snprintf(o->message, sizeof o->message, "%s", j.message.c_str());
  return MYCEL_OK;
}

extern "C" int32_t mycel_server_wait(mycel_server* s, int64_t id, double timeout_s) {
  if (!s) return mycel::set_error(nullptr, MYCEL_E_ARG, "NULL server");
  std::unique_lock<std::mutex> lk(s->m);
  auto finished = [&] {
    if (id >= 0) {
      auto it = s->jobs.find(id);
      return it == s->jobs.end() || it->second->state >= MYCEL_JOB_DONE;
    }
    for (auto& kv : s->jobs)
      if (kv.second->state < MYCEL_JOB_DONE) return false;
    return true;
  };
  if (id >= 0 && !s->jobs.count(id)) {
    s->last_error = "unknown job id";
    return MYCEL_E_ARG;
  }
  if (timeout_s < 0) {
    s->cv_done.wait(lk, finished);
    return MYCEL_OK;
  }
  if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), finished)) {
    s->last_error = "wait timed out";
    return MYCEL_E_TIMEOUT;
  }
  return MYCEL_OK;
}

extern "C" int32_t mycel_server_job_result(mycel_server* s, int64_t id, mycel_iter_record* history, int32_t cap,
                                           float* phys, float* des, double* u) {
  if (!s) return mycel::set_error(nullptr, MYCEL_E_ARG, "NULL server");
  std::lock_guard<std::mutex> lk(s->m);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) {
    s->last_error = "unknown job id";
    return MYCEL_E_ARG;
  }
  const Job& j = *it->second;
  if (j.state != MYCEL_JOB_DONE) {
    s->last_error = j.state == MYCEL_JOB_FAILED ? "job failed: " + j.message : "job has not finished";
    return j.state == MYCEL_JOB_FAILED ? j.status : MYCEL_E_INVALID_OPERATION;
  }
  if (history)
    for (int32_t q = 0; q < cap && q < (int32_t)j.history.size(); ++q) history[q] = j.history[(size_t)q];
  if (phys && !j.phys.empty()) std::memcpy(phys, j.phys.data(), sizeof(float) * j.phys.size());
  if (des && !j.des.empty()) std::memcpy(des, j.des.data(), sizeof(float) * j.des.size());
  if (u) {
    if (j.u.empty()) {
      s->last_error = "the job did not keep u";
      return MYCEL_E_INVALID_OPERATION;
    }
    std::memcpy(u, j.u.data(), sizeof(double) * j.u.size());
  }
  return MYCEL_OK;
}

extern "C" int32_t mycel_server_stats_get(mycel_server* s, mycel_server_stats* o) {
  if (!s || !o) return mycel::set_error(nullptr, MYCEL_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->m);
  std::memset(o, 0, sizeof *o);
  std::vector<double> lat, qd;
  double first = -1, last = 0, sum = 0;
  for (auto& kv : s->jobs) {
    const Job& j = *kv.second;
    ++o->submitted;
    if (first < 0 || j.t_submit < first) first = j.t_submit;
    if (j.state == MYCEL_JOB_QUEUED) ++o->queued;
    else if (j.state == MYCEL_JOB_RUNNING) ++o->running;
    else if (j.state == MYCEL_JOB_FAILED) ++o->failed;
    else {
      ++o->completed;
      o->simp_iterations += j.iterations;
      lat.push_back(j.t_finish - j.t_submit);
      qd.push_back(j.t_start - j.t_submit);
      sum += j.t_finish - j.t_submit;
      last = std::max(last, j.t_finish);
      o->max_latency_s = std::max(o->max_latency_s, j.t_finish - j.t_submit);
    }
  }
  o->first_submit_s = first < 0 ? 0 : first;
  o->last_finish_s = last;
  o->p50_latency_s = percentile(lat, 0.50);
  o->p99_latency_s = percentile(lat, 0.99);
  o->mean_latency_s = lat.empty() ? 0.0 : sum / (double)lat.size();
  o->p50_queue_s = percentile(qd, 0.50);
  o->p99_queue_s = percentile(qd, 0.99);
  o->admitted_bytes = s->admitted;
  o->peak_admitted_bytes = s->peak;
  return MYCEL_OK;
}

extern "C" int32_t mycel_server_destroy(mycel_server* s) {
  if (!s) return MYCEL_OK;
  {
    std::lock_guard<std::mutex> lk(s->m);
    for (Job* j : s->queue) {
      j->state = MYCEL_JOB_FAILED;
      j->status = MYCEL_E_CANCELLED;
      j->message = "server destroyed before the job started";
    }
    s->queue.clear();
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (mycel_ctx* c : s->ctxs) mycel_ctx_destroy(c);
  delete s;
  return MYCEL_OK;
}

extern "C" const char* mycel_server_last_error(mycel_server* s) {
  if (!s) return "NULL server";
  thread_local std::string copy;
  std::lock_guard<std::mutex> lk(s->m);
  copy = s->last_error;
  return copy.c_str();
}
