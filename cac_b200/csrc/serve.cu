// Serving: a job queue drained by worker threads, each owning one context
// (its own CUDA stream and device buffers, reused from job to job), so jobs
// of any size run concurrently on the GPU and start as soon as a worker and
// the HBM budget allow (continuous admission, first come first served).
//
// No reference counterpart: the reference runs one input deck per process.
// A job is one system and one command, `run N` with fix nve or `minimize`
// with the FIRE iterate, executed through the same context calls a single
// run makes, so its results do not depend on what else is being served.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cacb200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  int64_t id = 0;
  int kind = CACB200_JOB_NVE;
  double boxlo[3], boxhi[3];
  int na = 0, ne = 0;
  std::vector<double> x, v, nodex, nodev;
  double mass = 1.0;
  int steps = 0;          // NVE steps or FIRE iteration cap
  double dt = 0.001, etol = 0.0, ftol = 0.0;
  // NVE under fix langevin (cacb200_server_submit_nvt)
  bool langevin = false;
  double lgv_t0 = 0, lgv_t1 = 0, lgv_damp = 1;
  int lgv_seed = 1, lgv_zero = 0;
  size_t bytes = 0;       // device-memory estimate used for admission
  // results
  int status = 1;         // 1 queued, 2 running, then a CACB200_* code
  std::string error;
  double energy = 0.0;
  double thermo[CACB200_THERMO_N] = {};   // the job's last state, metal units
  int niter = 0, stop_code = -1;
  Clock::time_point t_submit, t_start, t_end;
};

struct PairConfig {
  int style = 0;          // 1 LJ, 2 EAM
  double eps = 0, sigma = 0, cut = 0;
  int nrho = 0, nr = 0;
  double drho = 0, dr = 0;
  std::vector<double> frho, rhor, z2r;
};

// Device bytes one job may hold: site table at full capacity (atoms, Gauss
// points, every lattice site; FP64 and the mixed copy), list slots for the
// starting capacity of 160 entries per i-site (raw, image, packed), state,
// forces and per-site work arrays.
size_t job_bytes(int na, int ne) {
  size_t nsi = (size_t)na + 8 * (size_t)ne;
  size_t ns = nsi + 729 * (size_t)ne;
  return 48 * ns + 9 * 160 * nsi + 200 * (size_t)na + 800 * (size_t)ne + (64u << 20);
}

}  // namespace

struct cacb200_server {
  int device = 0, nworkers = 1, precision = CACB200_FP64;
  double budget = 0.0;
  PairConfig pair;
  double skin = 1.0;
  int every = 10;
  int segment = 0;        // NVE jobs: restart from the job's initial state every `segment` steps (0: never)
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  std::deque<Job *> queue;
  std::map<int64_t, std::unique_ptr<Job>> jobs;
  int64_t next_id = 1;
  size_t in_use = 0;
  bool started = false, stopping = false;
  std::vector<std::thread> workers;
  std::string last_error;
};

namespace {

// Configure a worker's context for the server's pair style and settings.
int configure(cacb200_server *s, cacb200_ctx *c) {
  int rc = cacb200_set_precision(c, s->precision);
  if (rc) return rc;
  if (s->pair.style == 1) rc = cacb200_set_lj(c, s->pair.eps, s->pair.sigma, s->pair.cut);
  else
    rc = cacb200_set_eam(c, s->pair.nrho, s->pair.drho, s->pair.nr, s->pair.dr, s->pair.cut, s->pair.frho.data(),
                         s->pair.rhor.data(), s->pair.z2r.data());
  if (rc) return rc;
  return cacb200_set_neighbor(c, s->skin, s->every);
}

// One job on a worker's context; results into the job.
int execute(cacb200_ctx *c, Job &j, int segment) {
  int rc = cacb200_upload_system(c, j.boxlo, j.boxhi, j.na, j.x.data(), j.v.data(), j.ne, j.nodex.data(),
                                 j.nodev.data(), j.mass);
  if (rc) return rc;
  if (j.kind == CACB200_JOB_NVE) {
    const int seg = (segment > 0 && segment < j.steps) ? segment : j.steps;
    if (j.langevin) rc = cacb200_set_langevin(c, j.lgv_t0, j.lgv_t1, j.lgv_damp, j.lgv_seed, j.lgv_zero);
    if (!rc && seg < j.steps) rc = cacb200_snapshot(c);
    if (!rc) rc = cacb200_setup(c);
    for (int done = 0; !rc && done < j.steps;) {
      if (done > 0) {
        rc = cacb200_restore(c);
        if (!rc) rc = cacb200_setup(c);
        if (rc) break;
      }
      int k = std::min(seg, j.steps - done);
      done += k;
      const bool last = done == j.steps;
      rc = cacb200_run_nve(c, k, j.dt, last ? CACB200_ENERGY_GLOBAL : 0, last ? CACB200_VIRIAL_GLOBAL : 0);
    }
    // a run of 0 steps ends on the setup evaluation, which tallied both
    double vir[6];
    if (!rc) rc = cacb200_get_energy(c, &j.energy, vir, nullptr, nullptr, nullptr, nullptr);
    j.niter = j.steps;
  } else {
    double fnorm = 0.0;
    rc = cacb200_minimize_fire(c, j.etol, j.ftol, j.steps, j.dt, 1, &j.stop_code, &j.niter, &j.energy, &fnorm);
    // the minimiser tallies energies only: one more evaluation of the final
    // positions for the pressure (forces and energy unchanged)
    if (!rc) rc = cacb200_compute_forces(c, CACB200_ENERGY_GLOBAL, CACB200_VIRIAL_GLOBAL);
  }
  if (!rc) rc = cacb200_thermo(c, CACB200_UNITS_METAL, j.thermo);
  if (!rc) rc = cacb200_get_state(c, j.x.data(), j.v.data(), j.nodex.data(), j.nodev.data());
  return rc;
}

void worker(cacb200_server *s) {
  cacb200_ctx *c = nullptr;
  int rc = cacb200_ctx_create(s->device, &c);
  if (!rc) rc = configure(s, c);
  std::string setup_error = rc ? (c ? cacb200_last_error(c) : "no usable CUDA device") : "";
  std::unique_lock<std::mutex> lk(s->m);
  for (;;) {
    // first come first served: only the head of the queue may start, once it
    // fits the memory budget
    s->cv_work.wait(lk, [&] {
      return s->stopping ||
             (!s->queue.empty() && (double)(s->in_use + s->queue.front()->bytes) <= s->budget);
    });
    if (s->stopping) break;
    Job *j = s->queue.front();
    s->queue.pop_front();
    s->in_use += j->bytes;
    j->status = 2;
    j->t_start = Clock::now();
    lk.unlock();
    s->cv_work.notify_all();   // the next head may fit as well
    int jr = rc;
    std::string err = setup_error;
    if (!jr) {
      jr = execute(c, *j, s->segment);
      if (jr) err = cacb200_last_error(c);
    }
    lk.lock();
    j->t_end = Clock::now();
    j->status = jr;
    j->error = err;
    s->in_use -= j->bytes;
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
  lk.unlock();
  if (c) cacb200_ctx_destroy(c);
}

double seconds(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}

}  // namespace

extern "C" {

int cacb200_server_create(int device, int nworkers, double budget_bytes, int precision, cacb200_server **out) {
  if (!out || nworkers < 1 || nworkers > 256 || !(budget_bytes > 0.0) ||
      (precision != CACB200_FP64 && precision != CACB200_MIXED))
    return CACB200_EINVAL;
  auto *s = new cacb200_server;
  s->device = device;
  s->nworkers = nworkers;
  s->budget = budget_bytes;
  s->precision = precision;
  *out = s;
  return CACB200_OK;
}

int cacb200_server_set_lj(cacb200_server *s, double epsilon, double sigma, double cut) {
  if (!s) return CACB200_EINVAL;
  std::lock_guard<std::mutex> g(s->m);
  if (s->started) return CACB200_ESTATE;
  s->pair = PairConfig();
  s->pair.style = 1;
  s->pair.eps = epsilon;
  s->pair.sigma = sigma;
  s->pair.cut = cut;
  return CACB200_OK;
}

int cacb200_server_set_eam(cacb200_server *s, int nrho, double drho, int nr, double dr, double cut,
                           const double *frho, const double *rhor, const double *z2r) {
  if (!s || nrho < 5 || nr < 5 || !frho || !rhor || !z2r) return CACB200_EINVAL;
  std::lock_guard<std::mutex> g(s->m);
  if (s->started) return CACB200_ESTATE;
  s->pair = PairConfig();
  s->pair.style = 2;
  s->pair.nrho = nrho;
  s->pair.drho = drho;
  s->pair.nr = nr;
  s->pair.dr = dr;
  s->pair.cut = cut;
  s->pair.frho.assign(frho, frho + nrho);
  s->pair.rhor.assign(rhor, rhor + nr);
  s->pair.z2r.assign(z2r, z2r + nr);
  return CACB200_OK;
}

int cacb200_server_set_neighbor(cacb200_server *s, double skin, int every) {
  if (!s || !(skin >= 0.0) || every < 0) return CACB200_EINVAL;
  std::lock_guard<std::mutex> g(s->m);
  if (s->started) return CACB200_ESTATE;
  s->skin = skin;
  s->every = every;
  return CACB200_OK;
}

int cacb200_server_set_segment(cacb200_server *s, int segment) {
  if (!s || segment < 0) return CACB200_EINVAL;
  std::lock_guard<std::mutex> g(s->m);
  if (s->started) return CACB200_ESTATE;
  s->segment = segment;
  return CACB200_OK;
}

int cacb200_server_start(cacb200_server *s) {
  if (!s) return CACB200_EINVAL;
  std::lock_guard<std::mutex> g(s->m);
  if (s->started) return CACB200_ESTATE;
  if (s->pair.style == 0) {
    s->last_error = "no pair style set";
    return CACB200_ESTATE;
  }
  s->started = true;
  for (int k = 0; k < s->nworkers; k++) s->workers.emplace_back(worker, s);
  return CACB200_OK;
}

namespace {

int submit_job(cacb200_server *s, int kind, const double boxlo[3], const double boxhi[3], int natoms,
               const double *x, const double *v, int nelements, const double *nodex, const double *nodev,
               double mass, int steps, double dt, double etol, double ftol, const Job *thermostat,
               int64_t *job) {
  if (!s || !job) return CACB200_EINVAL;
  if ((kind != CACB200_JOB_NVE && kind != CACB200_JOB_FIRE) || !boxlo || !boxhi || natoms < 0 || nelements < 0 ||
      (natoms && (!x || !v)) || (nelements && (!nodex || !nodev)) || steps < 0 || !(dt > 0.0)) {
    std::lock_guard<std::mutex> g(s->m);
    s->last_error = "invalid job";
    return CACB200_EINVAL;
  }
  auto j = std::make_unique<Job>();
  j->kind = kind;
  for (int d = 0; d < 3; d++) {
    j->boxlo[d] = boxlo[d];
    j->boxhi[d] = boxhi[d];
  }
  j->na = natoms;
  j->ne = nelements;
  j->x.assign(x, x + 3 * (size_t)natoms);
  j->v.assign(v, v + 3 * (size_t)natoms);
  j->nodex.assign(nodex, nodex + 24 * (size_t)nelements);
  j->nodev.assign(nodev, nodev + 24 * (size_t)nelements);
  if (natoms == 0) j->x.resize(1), j->v.resize(1);
  if (nelements == 0) j->nodex.resize(1), j->nodev.resize(1);
  j->mass = mass;
  j->steps = steps;
  j->dt = dt;
  j->etol = etol;
  j->ftol = ftol;
  if (thermostat) {
    j->langevin = true;
    j->lgv_t0 = thermostat->lgv_t0;
    j->lgv_t1 = thermostat->lgv_t1;
    j->lgv_damp = thermostat->lgv_damp;
    j->lgv_seed = thermostat->lgv_seed;
    j->lgv_zero = thermostat->lgv_zero;
  }
  j->bytes = job_bytes(natoms, nelements);
  std::lock_guard<std::mutex> g(s->m);
  if (!s->started || s->stopping) {
    s->last_error = "server not running";
    return CACB200_ESTATE;
  }
  if ((double)j->bytes > s->budget) {
    s->last_error = "job larger than the server's memory budget";
    return CACB200_ENOMEM;
  }
  j->id = s->next_id++;
  j->t_submit = Clock::now();
  *job = j->id;
  s->queue.push_back(j.get());
  s->jobs[j->id] = std::move(j);
  s->cv_work.notify_all();
  return CACB200_OK;
}

}  // namespace

int cacb200_server_submit(cacb200_server *s, int kind, const double boxlo[3], const double boxhi[3], int natoms,
                          const double *x, const double *v, int nelements, const double *nodex,
                          const double *nodev, double mass, int steps, double dt, double etol, double ftol,
                          int64_t *job) {
  return submit_job(s, kind, boxlo, boxhi, natoms, x, v, nelements, nodex, nodev, mass, steps, dt, etol, ftol,
                    nullptr, job);
}

int cacb200_server_submit_nvt(cacb200_server *s, const double boxlo[3], const double boxhi[3], int natoms,
                              const double *x, const double *v, int nelements, const double *nodex,
                              const double *nodev, double mass, int steps, double dt, double t_start,
                              double t_stop, double damp, int seed, int zero, int64_t *job) {
  // the fix's own checks up front (FixLangevin::FixLangevin, fix_langevin.cpp:40-60)
  if (!(damp > 0.0) || seed <= 0 || seed > 900000000 || !(t_start >= 0.0) || !(t_stop >= 0.0)) {
    if (s) {
      std::lock_guard<std::mutex> g(s->m);
      s->last_error = "invalid fix langevin settings";
    }
    return CACB200_EINVAL;
  }
  Job t;
  t.lgv_t0 = t_start;
  t.lgv_t1 = t_stop;
  t.lgv_damp = damp;
  t.lgv_seed = seed;
  t.lgv_zero = zero;
  return submit_job(s, CACB200_JOB_NVE, boxlo, boxhi, natoms, x, v, nelements, nodex, nodev, mass, steps, dt, 0.0,
                    0.0, &t, job);
}

int cacb200_server_thermo(cacb200_server *s, int64_t job, double *out) {
  if (!s || !out) return CACB200_EINVAL;
  std::lock_guard<std::mutex> g(s->m);
  auto it = s->jobs.find(job);
  if (it == s->jobs.end()) {
    s->last_error = "unknown job";
    return CACB200_EINVAL;
  }
  Job *j = it->second.get();
  if (j->status > 0) return CACB200_ESTATE;
  if (j->status < 0) {
    s->last_error = j->error;
    return j->status;
  }
  std::memcpy(out, j->thermo, sizeof(j->thermo));
  return CACB200_OK;
}

int cacb200_server_wait(cacb200_server *s, int64_t job, double timeout_s) {
  if (!s) return CACB200_EINVAL;
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->jobs.find(job);
  if (it == s->jobs.end()) {
    s->last_error = "unknown job";
    return CACB200_EINVAL;
  }
  Job *j = it->second.get();
  auto done = [&] { return j->status <= 0; };
  if (timeout_s < 0) s->cv_done.wait(lk, done);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) return CACB200_ETIMEDOUT;
  if (j->status != 0) s->last_error = j->error;
  return j->status;
}

int cacb200_server_result(cacb200_server *s, int64_t job, double *x, double *v, double *nodex, double *nodev,
                          double *energy, int *niter, int *stop_code, double *times) {
  if (!s) return CACB200_EINVAL;
  std::lock_guard<std::mutex> g(s->m);
  auto it = s->jobs.find(job);
  if (it == s->jobs.end()) {
    s->last_error = "unknown job";
    return CACB200_EINVAL;
  }
  Job *j = it->second.get();
  if (j->status > 0) return CACB200_ESTATE;
  if (times) {
    times[0] = seconds(j->t_submit, j->t_start);
    times[1] = seconds(j->t_start, j->t_end);
    times[2] = seconds(j->t_submit, j->t_end);
  }
  if (j->status < 0) {
    s->last_error = j->error;
    return j->status;
  }
  if (x && j->na) std::memcpy(x, j->x.data(), sizeof(double) * 3 * j->na);
  if (v && j->na) std::memcpy(v, j->v.data(), sizeof(double) * 3 * j->na);
  if (nodex && j->ne) std::memcpy(nodex, j->nodex.data(), sizeof(double) * 24 * j->ne);
  if (nodev && j->ne) std::memcpy(nodev, j->nodev.data(), sizeof(double) * 24 * j->ne);
  if (energy) *energy = j->energy;
  if (niter) *niter = j->niter;
  if (stop_code) *stop_code = j->stop_code;
  return CACB200_OK;
}

int cacb200_server_release(cacb200_server *s, int64_t job) {
  if (!s) return CACB200_EINVAL;
  std::lock_guard<std::mutex> g(s->m);
  auto it = s->jobs.find(job);
  if (it == s->jobs.end()) return CACB200_EINVAL;
  if (it->second->status > 0) return CACB200_ESTATE;
  s->jobs.erase(it);
  return CACB200_OK;
}

const char *cacb200_server_last_error(const cacb200_server *s) {
  return s ? s->last_error.c_str() : "invalid server";
}

int cacb200_server_destroy(cacb200_server *s) {
  if (!s) return CACB200_EINVAL;
  {
    std::lock_guard<std::mutex> g(s->m);
    s->stopping = true;
    for (Job *j : s->queue) {
      j->status = CACB200_ESTATE;
      j->error = "server stopped before the job started";
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  for (auto &t : s->workers) t.join();
  delete s;
  return CACB200_OK;
}

}  // extern "C"
