// Many independent models (meshes of uneven size, one source each) stepped
// together: the adap_euler loop of every model in lockstep, with the
// triangular solves of all models of a step merged into one forward and one
// backward persistent kernel.
//
// Per model the host logic is that of the single-model time loop
// (src/FETD_FWD.f90:1229-1464): its own dt, refactorisations at the
// dt-doubling trials, accept/reject test and factor-slot ping-pong.  The
// models share the step counter, so their trials fall on the same steps;
// a model whose time has reached time_maximum drops out (its tasks are
// skipped by the merged kernels).  Everything else of a step (BDF2 SpMV,
// source, receivers) is launched per model on the batch stream, and a full
// dt segment is captured once as a CUDA graph when all models step it alike.
// The refactorisations at a trial run on the models' own streams at the same
// time.  The order in which the merged kernels claim tasks and the number of
// resident CTAs come from a small autotuner that times the candidates on the
// first step's factors.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <numeric>

#include "batch.h"
#include "factor.h"
#include "solve.h"

namespace temf {
namespace {

__global__ void k_set_ptr_b(double** p, double* v) { *p = v; }
__global__ void k_set_int_b(int* p, int v) { *p = v; }

struct ModelRun {
  temf_ctx* c = nullptr;
  RunResult* res = nullptr;
  int n = 0, nrec = 0, RS = 0;
  DBuf<double> ring, tmp, vco, err, coef, trace;
  DBuf<int> row_base;
  DBuf<double*> lptr;        // [0] slot 0, [1] slot 1, [2] current, [3] the other
  double* coef_h = nullptr;  // pinned
  double* err_h = nullptr;   // pinned
  // adap_euler state
  double time_cur = 0.0, step_cur = 0.0;
  int not_changed = 0, cur = 0, trace_rows = 0, trial_no = 0;
  bool running = true;
  struct Pending {
    int step;
    double t, dt, coef;
  };
  std::vector<Pending> pending;
  int seg_n = 0;  // normal steps flushed in the current segment

  double* E(int k) { return ring.p + (size_t)(((k % RS) + RS) % RS) * n; }
  double* T(int k) { return tmp.p + (size_t)k * n; }
  ~ModelRun() {
    if (coef_h) cudaFreeHost(coef_h);
    if (err_h) cudaFreeHost(err_h);
  }
};

struct BatchEngine {
  Batch& B;
  const RunOptions& opt;
  cudaStream_t st;
  int nm, dbl, dsz, nsite;
  std::vector<std::unique_ptr<ModelRun>> M;
  DBuf<SweepView> vf, vb;   // [site][model]
  DBuf<int> syncw;          // 2 claim counters, then per model 4*nsn+4 words
  DBuf<int> active;         // [site][model]
  int* act_h = nullptr;     // pinned copy of the table
  DBuf<int> errw;
  DBuf<int2> ordf, ordb;   // merged in-order (above-split) tasks
  // shared ready queues: [forward slots][backward slots][per-model backward
  // counts][fhead, bhead, ftail, btail]
  DBuf<int> gq;
  size_t gq_f = 0, gq_b = 0, gq_cnt = 0, gq_words = 0;
  std::vector<int> f_hi, b_lo, cnt_off;
  std::vector<std::vector<int>> finit_h, binit_h;
  struct InitSet {
    DBuf<int> f, b, tails;
    int nf = 0, nb = 0, qlim_f = 0, qlim_b = 0;
  };
  std::map<std::vector<int>, std::unique_ptr<InitSet>> init_sets;  // key: active flags
  int nf = 0, nb = 0, gridf = 0, gridb = 0;
  std::vector<std::vector<SolveTask>> ftask_h, btask_h;
  std::map<std::vector<int>, cudaGraphExec_t> graphs;  // key: N, then the participating models
  std::map<std::vector<int>, int64_t> graph_kernels;
  cudaEvent_t ev0, ev1;
  BatchStats& S;

  int site_normal(int k) const { return k - 1; }          // k = 1 .. dbl-1
  int site_fine(int i) const { return dbl - 1 + i; }       // i = 0 .. dsz-1
  int site_coarse() const { return dbl - 1 + dsz; }
  int site_tune() const { return dbl + dsz; }

  BatchEngine(Batch& b, const RunOptions& o) : B(b), opt(o), S(b.stats) {
    st = B.stream;
    nm = (int)B.models.size();
    dbl = opt.step_dble;
    dsz = opt.step_dblesize;
    nsite = dbl + dsz + 1;
    B.results.assign(nm, RunResult());
    f_hi.assign(nm, 0);
    b_lo.assign(nm, 0);
    cnt_off.assign(nm, 0);
    finit_h.resize(nm);
    binit_h.resize(nm);
    for (int m = 0; m < nm; ++m) {
      const temf_ctx& c = *B.models[m];
      queue_ranges(c, f_hi[m], b_lo[m]);
      queue_init_lists(c, finit_h[m], binit_h[m]);
      cnt_off[m] = (int)(gq_cnt);
      gq_f += f_hi[m];
      gq_b += c.splan.n_btask - b_lo[m];
      gq_cnt += c.splan.n_btask;
    }
    gq.alloc(gq_f + gq_b + gq_cnt + 4);
    gq_words = gq_f + gq_b + gq_cnt;
    std::vector<size_t> soff(nm);
    size_t words = 2;
    for (int m = 0; m < nm; ++m) {
      soff[m] = words;
      words += 4 * (size_t)B.models[m]->splan.nsn + 4;
    }
    syncw.alloc(words);
    active.alloc((size_t)nsite * nm);
    errw.alloc(1);
    TEMF_CUDA(cudaMemsetAsync(errw.p, 0, sizeof(int), st));
    TEMF_CUDA(cudaMallocHost((void**)&act_h, (size_t)nsite * nm * sizeof(int)));
    TEMF_CUDA(cudaEventCreate(&ev0));
    TEMF_CUDA(cudaEventCreate(&ev1));
    std::vector<SweepView> hf((size_t)nsite * nm), hb((size_t)nsite * nm);
    for (int m = 0; m < nm; ++m) {
      auto R = std::make_unique<ModelRun>();
      temf_ctx& c = *B.models[m];
      R->c = &c;
      R->res = &B.results[m];
      R->n = c.n_edges;
      R->nrec = c.rec.nrec;
      R->RS = dsz + 2;
      const size_t n = R->n;
      R->ring.alloc(n * R->RS);
      R->tmp.alloc(n * dsz);
      R->vco.alloc(n);
      R->err.alloc(two_error_len(1));
      R->coef.alloc(std::max(dbl, 8) + 8);
      R->trace.alloc((size_t)(dbl + 8) * std::max(R->nrec, 1) * 6);
      R->row_base.alloc(1);
      R->lptr.alloc(4);
      TEMF_CUDA(cudaMallocHost((void**)&R->coef_h, (std::max(dbl, 8) + 8) * sizeof(double)));
      TEMF_CUDA(cudaMallocHost((void**)&R->err_h, 2 * sizeof(double)));
      for (int s = 0; s < 2; ++s)
        if (c.slots[s].L.n < (size_t)slot_len(c)) c.slots[s].L.alloc(slot_len(c));
      ensure_update_buffer(c, 1);
      k_set_ptr_b<<<1, 1, 0, st>>>(R->lptr.p + 0, c.slots[0].L.p);
      k_set_ptr_b<<<1, 1, 0, st>>>(R->lptr.p + 1, c.slots[1].L.p);
      TEMF_CHECK_LAUNCH();
      int* sy = syncw.p + soff[m];
      for (int site = 0; site < nsite; ++site) {
        double* x = site < dbl - 1 ? R->E(site + 2)
                    : site < dbl - 1 + dsz ? R->T(site - (dbl - 1))
                                           : R->vco.p;
        double* const* Lb = R->lptr.p + (site == site_coarse() ? 3 : 2);
        SweepView a = fwd_view(c, Lb, x, sy), b = bwd_view(c, Lb, x, sy);
        const QueuePlan& Q = c.splan.q1;
        int* w = gq.p + gq_words;
        a.queue = gq.p;
        a.qhead = w + 0;
        a.qtail = w + 2;
        a.diag_task = Q.fdiag.p;
        a.q_lo = 0;
        a.q_hi = f_hi[m];
        a.tag = m << 24;
        b.queue = gq.p + gq_f;
        b.qhead = w + 1;
        b.qtail = w + 3;
        b.diag_task = Q.bdiag.p;
        b.dep_ptr = Q.bdep_ptr.p;
        b.dep = Q.bdep.p;
        b.need = Q.bneed.p;
        b.cnt = gq.p + gq_f + gq_b + cnt_off[m];
        b.q_lo = b_lo[m];
        b.q_hi = c.splan.n_btask;
        b.tag = m << 24;
        hf[(size_t)site * nm + m] = a;
        hb[(size_t)site * nm + m] = b;
      }
      // host copies of the task lists (for the merge orders)
      ftask_h.emplace_back(c.splan.n_ftask);
      btask_h.emplace_back(c.splan.n_btask);
      TEMF_CUDA(cudaMemcpy(ftask_h.back().data(), c.splan.ftask.p, c.splan.n_ftask * sizeof(SolveTask),
                           cudaMemcpyDeviceToHost));
      TEMF_CUDA(cudaMemcpy(btask_h.back().data(), c.splan.btask.p, c.splan.n_btask * sizeof(SolveTask),
                           cudaMemcpyDeviceToHost));
      M.push_back(std::move(R));
    }
    vf.upload(hf.data(), hf.size(), st);
    vb.upload(hb.data(), hb.size(), st);
    TEMF_CUDA(cudaStreamSynchronize(st));
    set_tuning(B.tune);
  }
  ~BatchEngine() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    if (act_h) cudaFreeHost(act_h);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
  }

  // --- merged task orders ----------------------------------------------------
  // Every order keeps each model's own task order, so a wait always targets a
  // task claimed earlier.
  std::vector<int2> merge(const std::vector<std::vector<SolveTask>>& tasks, int policy, bool forward) {
    std::vector<int2> out;
    size_t total = 0;
    for (auto& t : tasks) total += t.size();
    out.reserve(total);
    if (policy == 2) {
      for (int m = 0; m < nm; ++m)
        for (int i = 0; i < (int)tasks[m].size(); ++i) out.push_back(make_int2(m, i));
      return out;
    }
    struct Key {
      double k;
      int m, i;
    };
    std::vector<Key> keys;
    keys.reserve(total);
    for (int m = 0; m < nm; ++m) {
      const int nt = (int)tasks[m].size();
      const Symbolic& Sy = B.models[m]->sym;
      for (int i = 0; i < nt; ++i) {
        double k;
        if (policy == 0) {
          k = (i + 0.5) / nt;
        } else {
          // level counted from the leaves (forward) or from the root (backward)
          const int l = Sy.sn_level[tasks[m][i].s];
          k = forward ? l : (Sy.nlevels - 1 - l);
        }
        keys.push_back({k, m, i});
      }
    }
    std::stable_sort(keys.begin(), keys.end(), [](const Key& a, const Key& b) {
      return a.k < b.k || (a.k == b.k && a.m < b.m);
    });
    // a stable sort on (key, model) keeps each model's tasks in their order
    // only if the keys grow with i: true for policy 0; for policy 1 the
    // schedules are level-ordered (build_sched), so the keys do not decrease
    for (auto& k : keys) out.push_back(make_int2(k.m, k.i));
    return out;
  }

  void set_tuning(const BatchTuning& t) {
    // only the in-order tasks are merged; the queued ones go through the shared queue
    std::vector<std::vector<SolveTask>> fs(nm), bs(nm);
    for (int m = 0; m < nm; ++m) {
      fs[m].assign(ftask_h[m].begin() + f_hi[m], ftask_h[m].end());
      bs[m].assign(btask_h[m].begin(), btask_h[m].begin() + b_lo[m]);
    }
    auto of = merge(fs, t.order, true);
    auto ob = merge(bs, t.order, false);
    for (auto& v : of) v.y += f_hi[v.x];  // back to schedule indices
    nf = (int)of.size();
    nb = (int)ob.size();
    ordf.upload(of.data(), of.size(), st);
    ordb.upload(ob.data(), ob.size(), st);
    TEMF_CUDA(cudaStreamSynchronize(st));
    gridf = std::max(1, models_grid(true) * t.grid_pct / 100);
    gridb = std::max(1, models_grid(false) * t.grid_pct / 100);
  }

  // one merged solve of site `site` for the models flagged in its active row
  // initially ready queued tasks of an active set (cached: the set changes rarely)
  InitSet& init_set(const std::vector<int>& act) {
    auto it = init_sets.find(act);
    if (it != init_sets.end()) return *it->second;
    auto I = std::make_unique<InitSet>();
    std::vector<int> f, b;
    for (int m = 0; m < nm; ++m) {
      if (!act[m]) continue;
      for (int t : finit_h[m]) f.push_back((m << 24 | t) + 1);
      for (int t : binit_h[m]) b.push_back((m << 24 | t) + 1);
      I->qlim_f += f_hi[m];
      I->qlim_b += B.models[m]->splan.n_btask - b_lo[m];
    }
    I->nf = (int)f.size();
    I->nb = (int)b.size();
    if (f.empty()) I->f.alloc(1); else I->f.upload(f.data(), f.size(), st);
    if (b.empty()) I->b.alloc(1); else I->b.upload(b.data(), b.size(), st);
    const int tails[2] = {I->nf, I->nb};
    I->tails.upload(tails, 2, st);
    TEMF_CUDA(cudaStreamSynchronize(st));
    return *init_sets.emplace(act, std::move(I)).first->second;
  }

  void solve_site(int site) {
    std::vector<int> act(act_h + (size_t)site * nm, act_h + (size_t)(site + 1) * nm);
    InitSet& I = init_set(act);
    TEMF_CUDA(cudaMemsetAsync(syncw.p, 0, syncw.bytes(), st));
    TEMF_CUDA(cudaMemsetAsync(gq.p, 0, gq.bytes(), st));
    if (I.nf) TEMF_CUDA(cudaMemcpyAsync(gq.p, I.f.p, I.nf * sizeof(int), cudaMemcpyDeviceToDevice, st));
    if (I.nb) TEMF_CUDA(cudaMemcpyAsync(gq.p + gq_f, I.b.p, I.nb * sizeof(int), cudaMemcpyDeviceToDevice, st));
    TEMF_CUDA(cudaMemcpyAsync(gq.p + gq_words + 2, I.tails.p, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st));
    launch_solve_models(nf, ordf.p, vf.p + (size_t)site * nm, nb, ordb.p, vb.p + (size_t)site * nm,
                        active.p + (size_t)site * nm, syncw.p, errw.p, gridf, gridb, I.qlim_f, I.qlim_b, st);
    S.launches += 2;
    S.solves += 1;
  }

  void check_err() {
    int v = 0;
    TEMF_CUDA(cudaMemcpyAsync(&v, errw.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TEMF_CUDA(cudaStreamSynchronize(st));
    if (v) throw StateError("a merged triangular-solve wait timed out (code " + std::to_string(v) + ")");
  }

  double source_scalar(const ModelRun& R, int step_no, double t, double dt) const {
    if (step_no >= opt.step_dvsi) return 0.0;  // sys_right, src/FETD_FWD.f90:1484
    const Source& s = R.c->src;
    return 2.0 * dt * time_const_p(s.source_type, s.pulse_type, t, s.t0, s.current);
  }

  void out_row(ModelRun& R, int step_no, double t, double dt) {
    R.res->steps.push_back(step_no);
    R.res->times.push_back(t);
    R.res->dts.push_back(dt);
  }

  void sample(ModelRun& R, const double* x, int k) {
    if (!R.nrec) return;
    launch_receivers_row(*R.c, x, 1, R.row_base.p, k, R.trace.p, st);
    S.launches += 1;
  }

  void flush_trace(ModelRun& R) {
    if (R.trace_rows == 0) return;
    if (R.nrec) {
      const size_t cnt = (size_t)R.trace_rows * R.nrec * 6;
      const size_t off = R.res->samples.size();
      R.res->samples.resize(off + cnt);
      TEMF_CUDA(cudaMemcpyAsync(R.res->samples.data() + off, R.trace.p, cnt * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
      TEMF_CUDA(cudaStreamSynchronize(st));
    }
    R.trace_rows = 0;
  }

  void copy_vec(ModelRun& R, double* dst, const double* src) {
    if (dst != src)
      TEMF_CUDA(cudaMemcpyAsync(dst, src, (size_t)R.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }

  void set_current(ModelRun& R, int slot) {
    R.cur = slot;
    k_set_ptr_b<<<1, 1, 0, st>>>(R.lptr.p + 2, R.c->slots[slot].L.p);
    k_set_ptr_b<<<1, 1, 0, st>>>(R.lptr.p + 3, R.c->slots[1 - slot].L.p);
    TEMF_CHECK_LAUNCH();
  }

  // factorisations of several models, concurrently on their own streams
  void factor_models(const std::vector<std::pair<ModelRun*, std::pair<int, double>>>& jobs) {
    if (jobs.empty()) return;
    TEMF_CUDA(cudaStreamSynchronize(st));  // the models' streams read vectors the batch stream wrote
    const auto t0 = std::chrono::steady_clock::now();
    for (auto& j : jobs) launch_factor(*j.first->c, j.second.first, j.second.second);
    for (auto& j : jobs) {
      const int stt = finish_factor(*j.first->c, j.second.first);
      j.first->res->n_factor += 1;
      S.launches += 2 + 2 * (int64_t)j.first->c->sym.nlevels;
      if (stt != 0)
        throw StateError("non-positive pivot in a batched step-matrix factorisation at column " + std::to_string(stt));
    }
    S.ms_factor += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }

  // normal steps k = 1..N_m of every model from ring phase 0
  void flush() {
    std::vector<int> N(nm, 0);
    int Nmax = 0;
    bool any_src = false;
    for (int m = 0; m < nm; ++m) {
      N[m] = (int)M[m]->pending.size();
      Nmax = std::max(Nmax, N[m]);
      for (auto& p : M[m]->pending) any_src |= (p.coef != 0.0);
    }
    if (!Nmax) return;
    for (int k = 1; k <= Nmax; ++k)
      for (int m = 0; m < nm; ++m) act_h[(size_t)site_normal(k) * nm + m] = (k <= N[m]) ? 1 : 0;
    TEMF_CUDA(cudaMemcpyAsync(active.p, act_h, (size_t)(dbl - 1) * nm * sizeof(int), cudaMemcpyHostToDevice, st));
    for (int m = 0; m < nm; ++m) {
      ModelRun& R = *M[m];
      if (!N[m]) continue;
      k_set_int_b<<<1, 1, 0, st>>>(R.row_base.p, R.trace_rows);
      TEMF_CHECK_LAUNCH();
      if (any_src) {
        for (int k = 0; k < N[m]; ++k) R.coef_h[k] = R.pending[k].coef;
        TEMF_CUDA(cudaMemcpyAsync(R.coef.p, R.coef_h, N[m] * sizeof(double), cudaMemcpyHostToDevice, st));
      }
    }
    TEMF_CUDA(cudaEventRecord(ev0, st));
    bool uniform = true;
    for (int m = 0; m < nm; ++m) uniform &= (N[m] == 0 || N[m] == Nmax);
    auto body = [&]() {
      for (int k = 1; k <= Nmax; ++k) {
        for (int m = 0; m < nm; ++m) {
          if (k > N[m]) continue;
          ModelRun& R = *M[m];
          launch_bdf_rhs(*R.c, R.E(k), R.E(k - 1), R.E(k + 1), 1, st);
          S.launches += 1;
          if (any_src && R.pending[k - 1].coef != 0.0) {
            launch_source(*R.c, R.coef.p + (k - 1), R.E(k + 1), 1, st);
            S.launches += 1;
          }
        }
        solve_site(site_normal(k));
        for (int m = 0; m < nm; ++m)
          if (k <= N[m]) sample(*M[m], M[m]->E(k + 1), k - 1);
      }
    };
    if (opt.use_graphs && !any_src && uniform) {
      std::vector<int> key{Nmax};
      for (int m = 0; m < nm; ++m) key.push_back(N[m] ? 1 : 0);
      auto it = graphs.find(key);
      if (it == graphs.end()) {
        const int64_t l0 = S.launches, s0 = S.solves;
        cudaGraph_t g;
        TEMF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        body();
        TEMF_CUDA(cudaStreamEndCapture(st, &g));
        cudaGraphExec_t ge;
        TEMF_CUDA(cudaGraphInstantiate(&ge, g, 0));
        TEMF_CUDA(cudaGraphDestroy(g));
        graph_kernels[key] = S.launches - l0;
        S.launches = l0;
        S.solves = s0;
        it = graphs.emplace(key, ge).first;
      }
      TEMF_CUDA(cudaGraphLaunch(it->second, st));
      S.launches += graph_kernels[key];
      S.solves += Nmax;
    } else {
      body();
    }
    TEMF_CUDA(cudaEventRecord(ev1, st));
    TEMF_CUDA(cudaEventSynchronize(ev1));
    float ms = 0;
    TEMF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    S.ms_steps += ms;
    for (int m = 0; m < nm; ++m) {
      ModelRun& R = *M[m];
      for (auto& p : R.pending) out_row(R, p.step, p.t, p.dt);
      R.trace_rows += N[m];
      R.res->n_solve += N[m];
      R.seg_n = N[m];
      R.pending.clear();
    }
  }

  // the dt-doubling trial of every model in `P` (src/FETD_FWD.f90:1312-1421)
  void trial(const std::vector<int>& P, int step) {
    std::vector<const double*> a2(nm), a3(nm);
    for (int m : P) {
      ModelRun& R = *M[m];
      const int last = R.seg_n + 1, prev = R.seg_n;
      a2[m] = R.E(last);
      a3[m] = R.E(prev);
      double tt = R.time_cur;
      for (int i = 0; i < dsz; ++i) {
        R.coef_h[i] = source_scalar(R, step, tt, R.step_cur);
        tt += R.step_cur;
      }
      TEMF_CUDA(cudaMemcpyAsync(R.coef.p, R.coef_h, dsz * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    std::fill(act_h, act_h + (size_t)nsite * nm, 0);
    for (int m : P) {
      for (int i = 0; i < dsz; ++i) act_h[(size_t)site_fine(i) * nm + m] = 1;
      act_h[(size_t)site_coarse() * nm + m] = 1;
    }
    TEMF_CUDA(cudaMemcpyAsync(active.p + (size_t)site_fine(0) * nm, act_h + (size_t)site_fine(0) * nm,
                              (size_t)(dsz + 1) * nm * sizeof(int), cudaMemcpyHostToDevice, st));
    TEMF_CUDA(cudaEventRecord(ev0, st));
    for (int i = 0; i < dsz; ++i) {
      for (int m : P) {
        ModelRun& R = *M[m];
        launch_bdf_rhs(*R.c, a2[m], a3[m], R.T(i), 1, st);
        S.launches += 1;
        if (R.coef_h[i] != 0.0) { launch_source(*R.c, R.coef.p + i, R.T(i), 1, st); S.launches += 1; }
      }
      solve_site(site_fine(i));
      for (int m : P) {
        a3[m] = a2[m];
        a2[m] = M[m]->T(i);
        M[m]->res->n_solve += 1;
      }
    }
    TEMF_CUDA(cudaEventRecord(ev1, st));
    TEMF_CUDA(cudaEventSynchronize(ev1));
    float ms = 0;
    TEMF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    S.ms_steps += ms;
    // coarse step with dsz*dt from the history, in the other factor slot
    std::vector<std::pair<ModelRun*, std::pair<int, double>>> jobs;
    for (int m : P) jobs.push_back({M[m].get(), {1 - M[m]->cur, M[m]->step_cur * dsz}});
    factor_models(jobs);
    TEMF_CUDA(cudaEventRecord(ev0, st));
    for (int m : P) {
      ModelRun& R = *M[m];
      const int last = R.seg_n + 1;
      const double tmp_step = R.step_cur * dsz;
      const double tmp_time = R.time_cur - R.step_cur + tmp_step;
      R.coef_h[dsz] = source_scalar(R, step, tmp_time, tmp_step);
      TEMF_CUDA(cudaMemcpyAsync(R.coef.p + dsz, R.coef_h + dsz, sizeof(double), cudaMemcpyHostToDevice, st));
      launch_bdf_rhs(*R.c, R.E(last), R.E(last - dsz), R.vco.p, 1, st);
      S.launches += 1;
      if (R.coef_h[dsz] != 0.0) { launch_source(*R.c, R.coef.p + dsz, R.vco.p, 1, st); S.launches += 1; }
    }
    solve_site(site_coarse());
    for (int m : P) {
      ModelRun& R = *M[m];
      launch_two_error(*R.c, R.vco.p, R.T(dsz - 1), 1, R.err.p, st);
      S.launches += 2;
      TEMF_CUDA(cudaMemcpyAsync(R.err_h, R.err.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
      R.res->n_solve += 1;
    }
    TEMF_CUDA(cudaEventRecord(ev1, st));
    TEMF_CUDA(cudaEventSynchronize(ev1));
    TEMF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    S.ms_steps += ms;
    check_err();
    for (int m : P) {
      ModelRun& R = *M[m];
      const int last = R.seg_n + 1;
      const double error = std::sqrt(R.err_h[0]) / std::sqrt(R.err_h[1]);
      const bool reject = error > 1.0e-4 && R.not_changed < 2;  // :1382
      R.trial_no++;
      R.res->trial_err.push_back(error);
      R.res->trial_acc.push_back(reject ? 0 : 1);
      k_set_int_b<<<1, 1, 0, st>>>(R.row_base.p, R.trace_rows);
      TEMF_CHECK_LAUNCH();
      if (reject) {
        sample(R, R.T(0), 0);
        out_row(R, step, R.time_cur, R.step_cur);
        copy_vec(R, R.E(0), R.E(last));
        copy_vec(R, R.E(1), R.T(0));
        R.not_changed += 1;
      } else {
        sample(R, R.T(dsz - 1), 0);
        copy_vec(R, R.E(0), opt.legacy_linux ? R.E(last - dsz) : R.E(last));
        copy_vec(R, R.E(1), R.T(dsz - 1));
        set_current(R, 1 - R.cur);
        R.time_cur = R.time_cur - R.step_cur + R.step_cur * dsz + (opt.legacy_linux ? R.step_cur : 0.0);
        R.step_cur = R.step_cur * dsz;
        out_row(R, step, R.time_cur, R.step_cur);
        R.not_changed = 0;
      }
      R.trace_rows += 1;
      flush_trace(R);
      R.seg_n = 0;
    }
  }

  // time the candidate schedules on one merged solve and keep the fastest
  void autotune() {
    const auto t0 = std::chrono::steady_clock::now();
    for (int m = 0; m < nm; ++m) act_h[(size_t)site_tune() * nm + m] = 1;
    TEMF_CUDA(cudaMemcpyAsync(active.p + (size_t)site_tune() * nm, act_h + (size_t)site_tune() * nm,
                              nm * sizeof(int), cudaMemcpyHostToDevice, st));
    // a right-hand side that keeps the solves finite: the ones vector
    for (int m = 0; m < nm; ++m) {
      std::vector<double> one(M[m]->n, 1.0);
      TEMF_CUDA(cudaMemcpyAsync(M[m]->vco.p, one.data(), one.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    const int orders[3] = {0, 1, 2};
    const int grids[2] = {100, 67};
    BatchTuning best = B.tune;
    double best_ms = 1e30;
    S.tune_ms.clear();
    for (int o : orders)
      for (int g : grids) {
        BatchTuning t;
        t.order = o;
        t.grid_pct = g;
        set_tuning(t);
        solve_site(site_tune());  // warm-up
        TEMF_CUDA(cudaEventRecord(ev0, st));
        for (int r = 0; r < 3; ++r) solve_site(site_tune());
        TEMF_CUDA(cudaEventRecord(ev1, st));
        TEMF_CUDA(cudaEventSynchronize(ev1));
        float ms = 0;
        TEMF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        S.tune_ms.push_back(ms / 3.0);
        if (ms < best_ms) { best_ms = ms; best = t; }
      }
    check_err();
    B.tune = best;
    B.tuned = true;
    set_tuning(best);
    S.ms_tune = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }

  void run(bool tune) {
    TEMF_CUDA(cudaEventRecord(ev0, st));
    const auto t_start = std::chrono::steady_clock::now();
    const double limit = opt.time_maximum;
    for (auto& R : M) R->step_cur = R->c->src.t0 / opt.step_dvsi;  // time_solver, src/FETD_FWD.f90:1188
    int step = 0;
    for (;;) {
      bool any = false;
      for (auto& R : M) {
        if (R->running && !(R->time_cur < limit)) R->running = false;
        if (R->running && opt.max_steps > 0 && step >= opt.max_steps) R->running = false;
        any |= R->running;
      }
      if (!any) break;
      step += 1;
      std::vector<int> P;
      for (int m = 0; m < nm; ++m)
        if (M[m]->running) {
          M[m]->time_cur += M[m]->step_cur;
          P.push_back(m);
        }
      if (step == 1) {
        std::vector<std::pair<ModelRun*, std::pair<int, double>>> jobs;
        for (int m : P) {
          ModelRun& R = *M[m];
          TEMF_CUDA(cudaMemsetAsync(R.E(1), 0, (size_t)R.n * sizeof(double), st));
          TEMF_CUDA(cudaMemsetAsync(R.E(0), 0, (size_t)R.n * sizeof(double), st));
          k_set_int_b<<<1, 1, 0, st>>>(R.row_base.p, 0);
          TEMF_CHECK_LAUNCH();
          R.trace_rows = 0;
          sample(R, R.E(1), 0);
          out_row(R, 0, R.time_cur - R.step_cur, R.step_cur);
          R.trace_rows = 1;
          jobs.push_back({&R, {0, R.step_cur}});
        }
        factor_models(jobs);
        for (int m : P) set_current(*M[m], 0);
        if (tune && !B.tuned) autotune();
      }
      if (step % dbl == 0) {
        flush();
        trial(P, step);
        continue;
      }
      for (int m : P) {
        ModelRun& R = *M[m];
        R.pending.push_back({step, R.time_cur, R.step_cur, source_scalar(R, step, R.time_cur, R.step_cur)});
        if (R.trace_rows + (int)R.pending.size() >= dbl + 6) throw StateError("receiver trace overflow");
      }
    }
    flush();
    for (auto& R : M) flush_trace(*R);
    check_err();
    TEMF_CUDA(cudaEventRecord(ev1, st));
    TEMF_CUDA(cudaEventSynchronize(ev1));
    S.steps = step;
    S.ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    for (auto& R : M) {
      R->res->ms_total = S.ms_total;
      R->res->ms_steps = S.ms_steps;
      R->res->ms_factor = S.ms_factor;
      R->res->launches = S.launches;
    }
  }
};

}  // namespace

void run_batch(Batch& B, const RunOptions& opt, bool autotune) {
  if (B.models.empty()) throw ArgError("empty batch");
  if (opt.step_dvsi <= 0 || opt.step_dble <= 0 || !(opt.time_maximum > 0))
    throw ArgError("sp_division, sp_double and time_maximum must be positive");
  if (opt.step_dblesize < 2 || opt.step_dblesize > 8) throw ArgError("sp_dblesize must be in [2, 8]");
  if (opt.step_dble < opt.step_dblesize + 2)
    throw ArgError("sp_double must be at least sp_dblesize + 2 (the coarse trial step reads the history)");
  for (temf_ctx* c : B.models) {
    if (c->device != B.device) throw ArgError("all models of a batch must be on the batch's device");
    if (std::max(1, c->src.nrhs) != 1) throw ArgError("batched models take one right-hand side each");
    if (c->src.pulse_type == 3) throw ArgError("batched models run from rest (pulse types 1 and 2)");
  }
  if (B.models.size() > 127) throw ArgError("a batch holds at most 127 models");
  for (temf_ctx* c : B.models)
    if (c->splan.n_ftask >= (1 << 24) || c->splan.n_btask >= (1 << 24))
      throw ArgError("a batched model has too many solve tasks (2^24)");
  const std::vector<double> tuned_ms = B.stats.tune_ms;  // keep the last tuning's candidate times
  B.stats = BatchStats();
  B.stats.tune_ms = tuned_ms;
  BatchEngine eng(B, opt);
  eng.run(autotune);
  for (temf_ctx* c : B.models) c->slots[0].valid = c->slots[1].valid = false;
}

}  // namespace temf
