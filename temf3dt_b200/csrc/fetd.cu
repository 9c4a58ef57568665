// The FETD time loop on the GPU: adaptive BDF2 with dt-doubling trials.
//
// Host logic follows adap_euler (src/FETD_FWD.f90:1229-1464) step for step:
// the time bookkeeping, the trial at every sp_double-th step (two fine steps
// with dt against one coarse step with sp_dblesize*dt from the history), the
// 1e-4 relative-L2 acceptance test with at most two consecutive rejections,
// and the factor-slot ping-pong.  Everything between two trials runs on the
// device: the sp_double-1 normal steps of a segment (SpMV -> solve ->
// receivers) are captured once as a CUDA graph and replayed for every
// segment whose source term is zero; the factor slot in use is read through a
// device-side pointer so the same graph serves both slots.  The host reads
// back two scalars per trial (the error test) and the receiver samples of
// the segment.
#include <cmath>
#include <map>

#include "element.cuh"
#include "factor.h"
#include "fetd.h"
#include "solve.h"

namespace temf {

// --- source waveforms (source_mod, src/FETD_UTILITY.f90:1030-1165) -----------
static double erfstepon1(double t, double t0) {  // :1088-1093
  return (1.0 / std::sqrt(3.141592653589793) * std::exp(1.0 / (t0 * t0) * (t - t0 / 2.0) * (t - t0 / 2.0) * (-25.0)) *
          5.0) / t0;
}
static double deltafunc1(double t, double t0) {  // :1144-1147
  const double a = t * 5.436563656918091 - t0 * 2.718281828459046;
  return -1.0 / (t0 * t0) * std::exp(-1.0 / (t0 * t0) * a * a) * (t * 59.11244879144521 - t0 * 29.55622439572261);
}
double time_const_p(int source_type, int pulse_type, double t, double t0, double cur) {  // :1050-1078
  if (source_type == 1 && pulse_type == 1) return erfstepon1(t, t0) * cur;
  if (source_type == 1 && pulse_type == 2) return deltafunc1(t, t0) * cur;
  if (source_type == 1 && pulse_type == 3) return -erfstepon1(t, t0) * cur;
  throw ArgError("no such kind of source (source_type/pulse_type)");
}

__global__ void k_set_int(int* p, int v) { *p = v; }
__global__ void k_set_ptr(double** p, double* v) { *p = v; }

__global__ void k_receivers_row(int nrec, const int* __restrict__ edges, const int* __restrict__ rrhs,
                                const double* __restrict__ w, const double* __restrict__ x, int nrhs,
                                const int* __restrict__ row_base, int k, double* __restrict__ trace) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrec * 6) return;
  const int rec = t / 6, q = t % 6;
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < 6; ++j) acc += w[rec * 36 + q * 6 + j] * x[(int64_t)edges[rec * 6 + j] * nrhs + rrhs[rec]];
  trace[((int64_t)(row_base[0] + k) * nrec + rec) * 6 + q] = acc;
}

void launch_receivers_row(temf_ctx& c, const double* x, int nrhs, const int* row_base, int k, double* trace,
                          cudaStream_t st) {
  const int nrec = c.rec.nrec;
  if (!nrec) return;
  k_receivers_row<<<ceil_div(nrec * 6, 128), 128, 0, st>>>(nrec, c.rec.d_edges.p, c.rec.d_rhs.p, c.rec.d_w.p, x, nrhs,
                                                           row_base, k, trace);
  TEMF_CHECK_LAUNCH();
}

// vtk_field_save (src/FETD_FWD.f90:1659-1711) for one output row: E and D of
// x (permuted order, one column) at every tet centroid and B += D dt; a row
// whose trigger bits are set (trig[row_base + k]) copies E, D, B into those
// snapshots (msh_output's data, :1790-1860).
__global__ void k_mesh_fields(int T, const double* __restrict__ xyz, const int* __restrict__ tet_vex,
                              const int* __restrict__ edges, const int* __restrict__ drc,
                              const double* __restrict__ x, const double* __restrict__ dt,
                              const int* __restrict__ trig, const int* __restrict__ row_base, int k,
                              double* __restrict__ b, double* __restrict__ snap, int nsnap) {
  const int mask = trig[row_base[0] + k];
  const double h = dt[0];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
    double X[4][3], ev[6], E[3], D[3];
    for (int v = 0; v < 4; ++v) {
      const int node = tet_vex[4 * (int64_t)t + v];
      for (int a = 0; a < 3; ++a) X[v][a] = xyz[3 * (int64_t)node + a];
    }
    for (int j = 0; j < 6; ++j) ev[j] = drc[6 * (int64_t)t + j] * x[edges[6 * (int64_t)t + j]];
    centroid_fields(X, ev, E, D);
    double B[3];
    for (int a = 0; a < 3; ++a) {
      B[a] = b[3 * (int64_t)t + a] + D[a] * h;
      b[3 * (int64_t)t + a] = B[a];
    }
    if (mask)
      for (int i = 0; i < nsnap; ++i)
        if ((mask >> i) & 1) {
          double* o = snap + ((int64_t)i * T + t) * 9;
          for (int a = 0; a < 3; ++a) {
            o[a] = E[a];
            o[3 + a] = D[a];
            o[6 + a] = B[a];
          }
        }
  }
}

namespace {

struct Engine {
  temf_ctx& c;
  const RunOptions& opt;
  RunResult& res;
  cudaStream_t st;
  int n, nrhs, nrec, dbl, dsz, RS;
  DBuf<double> ring, tmp, vco, err, coef, trace, res_e;
  DBuf<int> row_base;
  DBuf<double*> lptr;  // [0] slot0, [1] slot1, [2] current
  double* coef_h = nullptr;
  double* err_h = nullptr;
  std::map<int, cudaGraphExec_t> graphs;
  std::map<int, int64_t> graph_kernels;
  cudaEvent_t ev0, ev1;
  int trace_rows = 0;
  int trial_no = 0;
  int cur = 0;
  // bookkeeping of one pass
  int pass_sign = 1;
  bool pass_output = true;
  // adjoint recording (eager launches only)
  bool rec = false;
  int W = 0;
  std::vector<int> slot_node, tnode;
  DBuf<double> recent;  // W most recent node states, node id % W
  int last_node = 0;
  // whole-mesh fields: active in the output pass until every snapshot is taken
  bool mf_act = false;
  int* mf_h = nullptr;        // pinned: trigger bits of the rows about to be sampled
  double* mf_dt_h = nullptr;  // pinned: their dt

  Engine(temf_ctx& c_, const RunOptions& o, RunResult& r) : c(c_), opt(o), res(r) {
    st = c.stream;
    n = c.n_edges;
    nrhs = std::max(1, c.src.nrhs);
    nrec = c.rec.nrec;
    dbl = opt.step_dble;
    dsz = opt.step_dblesize;
    RS = dsz + 2;
    const size_t vec = (size_t)n * nrhs;
    ring.alloc(vec * RS);
    tmp.alloc(vec * dsz);
    vco.alloc(vec);
    err.alloc(two_error_len(nrhs));
    coef.alloc(std::max(dbl, 8) + 8);
    trace.alloc((size_t)(dbl + 8) * std::max(nrec, 1) * 6);
    res_e.alloc(vec);
    row_base.alloc(1);
    lptr.alloc(3);
    TEMF_CUDA(cudaMallocHost((void**)&coef_h, (std::max(dbl, 8) + 8) * sizeof(double)));
    TEMF_CUDA(cudaMallocHost((void**)&err_h, 2 * nrhs * sizeof(double)));
    TEMF_CUDA(cudaEventCreate(&ev0));
    TEMF_CUDA(cudaEventCreate(&ev1));
    ensure_update_buffer(c, nrhs);
    for (int s = 0; s < 2; ++s)
      if (c.slots[s].L.n < (size_t)slot_len(c)) c.slots[s].L.alloc(slot_len(c));
    k_set_ptr<<<1, 1, 0, st>>>(lptr.p + 0, c.slots[0].L.p);
    k_set_ptr<<<1, 1, 0, st>>>(lptr.p + 1, c.slots[1].L.p);
    TEMF_CHECK_LAUNCH();
    if (c.mf.n() > 0) {
      if (nrhs != 1) throw ArgError("whole-mesh field dumps need one right-hand side");
      c.mf.trig.alloc(dbl + 8);
      c.mf.dt.alloc(1);
      TEMF_CUDA(cudaMallocHost((void**)&mf_h, (dbl + 8) * sizeof(int)));
      TEMF_CUDA(cudaMallocHost((void**)&mf_dt_h, sizeof(double)));
    }
    rec = opt.record_every > 0;
    if (rec) {
      if (nrhs != 1) throw ArgError("adjoint recording supports one right-hand side");
      if (c.src.pulse_type == 3) throw ArgError("adjoint recording covers runs from rest (pulse types 1 and 2)");
      // a node reads states at most 2*dsz+1 nodes back (the restart after an
      // accepted trial in the legacy schedule); the window covers that
      W = 2 * dsz + 2;
      recent.alloc(vec * W);
      slot_node.assign(RS, 0);
      tnode.assign(dsz, 0);
      AdjointRecord& A = c.adj;
      A.every = opt.record_every;
      A.valid = false;
      A.W = W;
      A.dt.clear(); A.coef.clear(); A.a.clear(); A.b.clear(); A.row_node.clear();
      A.ck_first.clear(); A.ck.clear();
    }
  }

  // --- recording helpers ---------------------------------------------------
  double* recent_slot(int node) { return recent.p + (size_t)(node % W) * n; }
  // called before node `k` (= last_node + 1) is computed
  void maybe_checkpoint(double dt) {
    AdjointRecord& A = c.adj;
    const int k = last_node + 1;
    if (!(k == 1 || (k - 1) % A.every == 0 || dt != A.dt.back())) return;
    auto buf = std::make_unique<DBuf<double>>();
    buf->alloc((size_t)W * n);
    for (int w = 0; w < W; ++w) {
      const int node = k - W + w;
      double* dst = buf->p + (size_t)w * n;
      if (node <= 0) TEMF_CUDA(cudaMemsetAsync(dst, 0, (size_t)n * sizeof(double), st));
      else TEMF_CUDA(cudaMemcpyAsync(dst, recent_slot(node), (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    A.ck_first.push_back(k);
    A.ck.push_back(std::move(buf));
  }
  // record node (dt, coef, a, b) whose state is now in `x`
  int record_node(double dt, double cf, int na, int nb, const double* x) {
    AdjointRecord& A = c.adj;
    const int k = ++last_node;
    A.dt.push_back(dt); A.coef.push_back(cf); A.a.push_back(na); A.b.push_back(nb);
    TEMF_CUDA(cudaMemcpyAsync(recent_slot(k), x, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    return k;
  }
  int sn(int k) const { return slot_node[((k % RS) + RS) % RS]; }
  void set_sn(int k, int node) { slot_node[((k % RS) + RS) % RS] = node; }
  ~Engine() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    if (mf_h) cudaFreeHost(mf_h);
    if (mf_dt_h) cudaFreeHost(mf_dt_h);
    if (coef_h) cudaFreeHost(coef_h);
    if (err_h) cudaFreeHost(err_h);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
  }

  double* E(int k) { return ring.p + (size_t)(((k % RS) + RS) % RS) * n * nrhs; }
  double* T(int k) { return tmp.p + (size_t)k * n * nrhs; }

  void set_current(int slot) {
    cur = slot;
    k_set_ptr<<<1, 1, 0, st>>>(lptr.p + 2, c.slots[slot].L.p);
    TEMF_CHECK_LAUNCH();
  }

  double factor(int slot, double dt) {
    TEMF_CUDA(cudaEventRecord(ev0, st));
    const int stt = numeric_factor(c, slot, dt);
    TEMF_CUDA(cudaEventRecord(ev1, st));
    TEMF_CUDA(cudaEventSynchronize(ev1));
    float ms = 0;
    TEMF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    res.ms_factor += ms;
    res.n_factor += 1;
    res.launches += 2 + 2 * (int64_t)c.sym.nlevels;
    if (stt != 0)
      throw StateError("non-positive pivot in the step-matrix factorisation at column " + std::to_string(stt) +
                       " (dt = " + std::to_string(dt) + ")");
    return ms;
  }

  int64_t solve_launches() const { return solve_launch_count(c, nrhs); }  // subtree and persistent task kernels

  // one BDF2 step: out = A^{-1} (M (4 e2 - e3) - coef * s)
  void step(const double* e2, const double* e3, double* out, const double* coefp, double* const* Lb) {
    launch_bdf_rhs(c, e2, e3, out, nrhs, st);
    res.launches += 1;
    if (coefp) { launch_source(c, coefp, out, nrhs, st); res.launches += 1; }
    launch_solve(c, Lb, out, nrhs, st);
    res.launches += solve_launches();
    res.n_solve += 1;
  }
  void sample(const double* x, int k) {
    if (mf_act) {
      const int T = c.n_tets;
      k_mesh_fields<<<std::min(ceil_div(T, 256), 148 * 16), 256, 0, st>>>(
          T, c.d_xyz.p, c.d_tet_vex.p, c.mf.edges.p, c.d_tet_drc.p, x, c.mf.dt.p, c.mf.trig.p, row_base.p, k,
          c.mf.b.p, c.mf.snap.p, c.mf.n());
      TEMF_CHECK_LAUNCH();
      res.launches += 1;
    }
    if (!nrec) return;
    k_receivers_row<<<ceil_div(nrec * 6, 128), 128, 0, st>>>(nrec, c.rec.d_edges.p, c.rec.d_rhs.p, c.rec.d_w.p, x,
                                                             nrhs, row_base.p, k, trace.p);
    TEMF_CHECK_LAUNCH();
    res.launches += 1;
  }
  // trigger bits of the output rows first_row .. first_row + n - 1 (times t)
  // and their dt, uploaded before those rows are sampled; the first row at or
  // after each vtkout time takes its snapshot (src/FETD_FWD.f90:1646-1655)
  void mf_rows(int first_row, const double* t, int nrows, double dt) {
    if (!mf_act) return;
    std::vector<int>& done = c.mf.done;
    for (int r = 0; r < nrows; ++r) {
      int mask = 0;
      for (int i = 0; i < c.mf.n(); ++i)
        if (!done[i] && t[r] >= c.mf.times[i]) {
          mask |= 1 << i;
          done[i] = 1;
        }
      mf_h[r] = mask;
    }
    mf_dt_h[0] = dt;
    TEMF_CUDA(cudaMemcpyAsync(c.mf.trig.p + first_row, mf_h, nrows * sizeof(int), cudaMemcpyHostToDevice, st));
    TEMF_CUDA(cudaMemcpyAsync(c.mf.dt.p, mf_dt_h, sizeof(double), cudaMemcpyHostToDevice, st));
  }
  // after the rows are sampled: stop once every snapshot is taken
  void mf_after() {
    if (!mf_act) return;
    TEMF_CUDA(cudaStreamSynchronize(st));  // mf_h is rewritten by the next rows
    bool all = true;
    for (int d : c.mf.done) all = all && d;
    if (all) mf_act = false;
  }
  double source_scalar(int step_no, double t, double dt) {
    if (step_no >= opt.step_dvsi) return 0.0;  // sys_right, src/FETD_FWD.f90:1484
    return 2.0 * dt * pass_sign * time_const_p(c.src.source_type, c.src.pulse_type, t, c.src.t0, c.src.current);
  }

  struct Pending { int step; double t, dt, coef; };
  std::vector<Pending> pending;

  void out_row(int step_no, double t, double dt) {
    if (!pass_output) return;
    res.steps.push_back(step_no);
    res.times.push_back(t);
    res.dts.push_back(dt);
  }

  void flush_trace() {
    if (trace_rows == 0) return;
    if (pass_output && nrec) {
      const size_t cnt = (size_t)trace_rows * nrec * 6;
      const size_t off = res.samples.size();
      res.samples.resize(off + cnt);
      TEMF_CUDA(cudaMemcpyAsync(res.samples.data() + off, trace.p, cnt * sizeof(double), cudaMemcpyDeviceToHost, st));
      TEMF_CUDA(cudaStreamSynchronize(st));
    }
    trace_rows = 0;
  }

  // run the pending normal steps k = 1..N from ring phase 0
  int flush_steps() {
    const int N = (int)pending.size();
    if (!N) return 0;
    bool any_src = false;
    for (auto& p : pending) any_src |= (p.coef != 0.0);
    k_set_int<<<1, 1, 0, st>>>(row_base.p, trace_rows);
    TEMF_CHECK_LAUNCH();
    if (mf_act) {
      std::vector<double> tr(N);
      for (int k = 0; k < N; ++k) tr[k] = pending[k].t;
      mf_rows(trace_rows, tr.data(), N, pending[0].dt);
    }
    const bool mf_now = mf_act;
    const int key = 2 * N + (mf_now ? 1 : 0);  // graphs with and without the mesh-field launches
    TEMF_CUDA(cudaEventRecord(ev0, st));
    if (opt.use_graphs && !any_src && !rec) {
      auto it = graphs.find(key);
      if (it == graphs.end()) {
        const int64_t l0 = res.launches;
        const int s0 = res.n_solve;
        cudaGraph_t g;
        TEMF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int k = 1; k <= N; ++k) {
          step(E(k), E(k - 1), E(k + 1), nullptr, lptr.p + 2);
          sample(E(k + 1), k - 1);
        }
        TEMF_CUDA(cudaStreamEndCapture(st, &g));
        cudaGraphExec_t ge;
        TEMF_CUDA(cudaGraphInstantiate(&ge, g, 0));
        TEMF_CUDA(cudaGraphDestroy(g));
        graph_kernels[key] = res.launches - l0;
        res.launches = l0;
        res.n_solve = s0;
        it = graphs.emplace(key, ge).first;
      }
      TEMF_CUDA(cudaGraphLaunch(it->second, st));
      res.launches += graph_kernels[key];
      res.n_solve += N;
    } else {
      for (int k = 0; k < N; ++k) coef_h[k] = pending[k].coef;
      if (any_src)
        TEMF_CUDA(cudaMemcpyAsync(coef.p, coef_h, N * sizeof(double), cudaMemcpyHostToDevice, st));
      for (int k = 1; k <= N; ++k) {
        if (rec) maybe_checkpoint(pending[k - 1].dt);
        step(E(k), E(k - 1), E(k + 1), any_src ? coef.p + (k - 1) : nullptr, lptr.p + 2);
        sample(E(k + 1), k - 1);
        if (rec) {
          const int id = record_node(pending[k - 1].dt, pending[k - 1].coef, sn(k), sn(k - 1), E(k + 1));
          set_sn(k + 1, id);
          c.adj.row_node.push_back(id);
        }
      }
    }
    TEMF_CUDA(cudaEventRecord(ev1, st));
    TEMF_CUDA(cudaEventSynchronize(ev1));
    float ms = 0;
    TEMF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    res.ms_steps += ms;
    for (auto& p : pending) out_row(p.step, p.t, p.dt);
    trace_rows += N;
    pending.clear();
    mf_after();
    return N;
  }

  void copy_vec(double* dst, const double* src) {
    if (dst != src)
      TEMF_CUDA(cudaMemcpyAsync(dst, src, (size_t)n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }

  // One pass of adap_euler.  Returns the device pointer of the final e1.
  const double* pass(const double* init_e) {
    int step = 0;
    double time_cur = 0.0;
    int not_changed = 0;
    double step_cur = c.src.t0 / opt.step_dvsi;  // time_solver, src/FETD_FWD.f90:1188
    const double time_limit = opt.time_maximum;
    const double* e1 = nullptr;
    int N = 0;  // normal steps in the current segment (ring phase)
    while (time_cur < time_limit) {
      if (opt.max_steps > 0 && step >= opt.max_steps) break;
      step += 1;
      time_cur += step_cur;
      if (step == 1) {
        if (init_e) { copy_vec(E(1), init_e); copy_vec(E(0), init_e); }
        else {
          TEMF_CUDA(cudaMemsetAsync(E(1), 0, (size_t)n * nrhs * sizeof(double), st));
          TEMF_CUDA(cudaMemsetAsync(E(0), 0, (size_t)n * nrhs * sizeof(double), st));
        }
        k_set_int<<<1, 1, 0, st>>>(row_base.p, 0);
        trace_rows = 0;
        if (c.mf.n() > 0 && pass_output) {  // a new output pass: B from zero, no snapshot taken
          mf_act = true;
          c.mf.done.assign(c.mf.n(), 0);
          TEMF_CUDA(cudaMemsetAsync(c.mf.b.p, 0, c.mf.b.bytes(), st));
          const double t0 = time_cur - step_cur;
          mf_rows(0, &t0, 1, step_cur);
        }
        sample(E(1), 0);
        mf_after();
        out_row(0, time_cur - step_cur, step_cur);
        if (rec) {
          set_sn(1, 0); set_sn(0, 0);
          last_node = 0;
          TEMF_CUDA(cudaMemsetAsync(recent.p, 0, recent.bytes(), st));
          c.adj.row_node.push_back(0);
        }
        trace_rows = 1;
        cur = 0;
        factor(0, step_cur);
        set_current(0);
        // first solve on this analysis: pick the sweep schedule (once)
        if (!(nrhs > 1 ? c.splan.qm.tuned : c.splan.tree.tuned)) tune_solve(c, 0, nrhs);
        N = 0;
        e1 = E(1);
      }
      if (step % dbl == 0) {
        N = flush_steps();
        const int last = N + 1, prev = N;
        // fine steps with dt (e_veri_1), src/FETD_FWD.f90:1312-1349
        double tt = time_cur;
        const double* a2 = E(last);
        const double* a3 = E(prev);
        TEMF_CUDA(cudaEventRecord(ev0, st));
        for (int i = 0; i < dsz; ++i) {
          coef_h[i] = source_scalar(step, tt, step_cur);
          tt += step_cur;
        }
        TEMF_CUDA(cudaMemcpyAsync(coef.p, coef_h, dsz * sizeof(double), cudaMemcpyHostToDevice, st));
        int a2n = rec ? sn(last) : 0, a3n = rec ? sn(prev) : 0;
        for (int i = 0; i < dsz; ++i) {
          if (rec) maybe_checkpoint(step_cur);
          step_fn(a2, a3, T(i), coef_h[i] != 0.0 ? coef.p + i : nullptr, lptr.p + 2);
          if (rec) {
            tnode[i] = record_node(step_cur, coef_h[i], a2n, a3n, T(i));
            a3n = a2n;
            a2n = tnode[i];
          }
          a3 = a2;
          a2 = T(i);
        }
        TEMF_CUDA(cudaEventRecord(ev1, st));
        TEMF_CUDA(cudaEventSynchronize(ev1));
        float ms = 0;
        TEMF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        res.ms_steps += ms;
        // coarse step with dsz*dt from the history (e_veri_2), :1350-1371
        const double tmp_step_cur = step_cur * dsz;
        const double tmp_time_cur = time_cur - step_cur + tmp_step_cur;
        const int other = 1 - cur;
        factor(other, tmp_step_cur);
        coef_h[dsz] = source_scalar(step, tmp_time_cur, tmp_step_cur);
        TEMF_CUDA(cudaEventRecord(ev0, st));
        TEMF_CUDA(cudaMemcpyAsync(coef.p + dsz, coef_h + dsz, sizeof(double), cudaMemcpyHostToDevice, st));
        step_fn(E(last), E(last - dsz), vco.p, coef_h[dsz] != 0.0 ? coef.p + dsz : nullptr, lptr.p + other);
        launch_two_error(c, vco.p, T(dsz - 1), nrhs, err.p, st);
        res.launches += 2;
        TEMF_CUDA(cudaMemcpyAsync(err_h, err.p, 2 * nrhs * sizeof(double), cudaMemcpyDeviceToHost, st));
        TEMF_CUDA(cudaEventRecord(ev1, st));
        TEMF_CUDA(cudaEventSynchronize(ev1));
        TEMF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        res.ms_steps += ms;
        if (const int fl = solve_error_flag(c))
          throw StateError("a triangular-solve wait timed out (code " + std::to_string(fl) + ")");
        double error = 0.0;
        for (int q = 0; q < nrhs; ++q) {
          const double e = std::sqrt(err_h[2 * q]) / std::sqrt(err_h[2 * q + 1]);
          error = (q == 0 || e > error || std::isnan(e)) ? e : error;
        }
        bool reject = error > 1.0e-4 && not_changed < 2;  // :1382
        if (trial_no < opt.n_forced && opt.forced && opt.forced[trial_no] >= 0) reject = opt.forced[trial_no] == 0;
        trial_no++;
        if (pass_output) {
          res.trial_err.push_back(error);
          res.trial_acc.push_back(reject ? 0 : 1);
        }
        k_set_int<<<1, 1, 0, st>>>(row_base.p, trace_rows);
        if (reject) {
          mf_rows(trace_rows, &time_cur, 1, step_cur);
          sample(T(0), 0);
          mf_after();
          out_row(step, time_cur, step_cur);
          if (rec) {
            c.adj.row_node.push_back(tnode[0]);
            const int n0 = sn(last);
            set_sn(0, n0);
            set_sn(1, tnode[0]);
          }
          copy_vec(E(0), E(last));
          copy_vec(E(1), T(0));
          e1 = E(1);
          not_changed += 1;
        } else {
          {
            const double t_row = tmp_time_cur + (opt.legacy_linux ? step_cur : 0.0);
            mf_rows(trace_rows, &t_row, 1, tmp_step_cur);
          }
          sample(T(dsz - 1), 0);
          mf_after();
          // e3 = all_e(idx) (src/FETD_FWD.f90:1405); the build that wrote the
          // shipped LINUX/*.field files restarted from all_e(idx - sp_dblesize)
          if (rec) {
            c.adj.row_node.push_back(tnode[dsz - 1]);
            const int n0 = opt.legacy_linux ? sn(last - dsz) : sn(last);
            set_sn(0, n0);
            set_sn(1, tnode[dsz - 1]);
          }
          copy_vec(E(0), opt.legacy_linux ? E(last - dsz) : E(last));
          copy_vec(E(1), T(dsz - 1));
          e1 = E(0);
          set_current(other);
          time_cur = tmp_time_cur + (opt.legacy_linux ? step_cur : 0.0);
          step_cur = tmp_step_cur;
          out_row(step, time_cur, step_cur);
          not_changed = 0;
        }
        trace_rows += 1;
        flush_trace();
        k_set_int<<<1, 1, 0, st>>>(row_base.p, 0);
        N = 0;
        continue;
      }
      pending.push_back({step, time_cur, step_cur, source_scalar(step, time_cur, step_cur)});
      // the trace buffer holds one segment; flush early only if it would overflow
      if (trace_rows + (int)pending.size() >= dbl + 6) {
        // cannot happen with sp_double steps per segment; guard anyway
        throw StateError("receiver trace overflow");
      }
    }
    N = flush_steps();
    if (N) e1 = E(N + 1);
    flush_trace();
    if (const int fl = solve_error_flag(c))
      throw StateError("a triangular-solve wait timed out (code " + std::to_string(fl) + ")");
    return e1;
  }

  void step_fn(const double* e2, const double* e3, double* out, const double* coefp, double* const* Lb) {
    step(e2, e3, out, coefp, Lb);
  }

  void run() {
    cudaEvent_t a, b;
    TEMF_CUDA(cudaEventCreate(&a));
    TEMF_CUDA(cudaEventCreate(&b));
    TEMF_CUDA(cudaEventRecord(a, st));
    if (c.src.pulse_type == 3) {
      // DC pass with the negated turn-off source, no output (src/FETD_FWD.f90:1212-1215)
      pass_sign = -1;
      pass_output = false;
      const double* e = pass(nullptr);
      copy_vec(res_e.p, e);
      pass_sign = 1;
      pass_output = true;
      trial_no = 0;
      pass(res_e.p);
    } else {
      pass_sign = 1;
      pass_output = true;
      pass(nullptr);
    }
    TEMF_CUDA(cudaEventRecord(b, st));
    TEMF_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    TEMF_CUDA(cudaEventElapsedTime(&ms, a, b));
    res.ms_total = ms;
    if (rec) c.adj.valid = true;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

}  // namespace

void run_fetd(temf_ctx& c, const RunOptions& opt, RunResult& res) {
  if (opt.step_dvsi <= 0 || opt.step_dble <= 0 || !(opt.time_maximum > 0))
    throw ArgError("sp_division, sp_double and time_maximum must be positive");
  if (opt.step_dblesize < 2 || opt.step_dblesize > 8) throw ArgError("sp_dblesize must be in [2, 8]");
  if (opt.step_dble < opt.step_dblesize + 2)
    throw ArgError("sp_double must be at least sp_dblesize + 2 (the coarse trial step reads the history)");
  res = RunResult();
  clear_solve_error_flag(c);
  Engine eng(c, opt, res);
  eng.run();
}

}  // namespace temf
