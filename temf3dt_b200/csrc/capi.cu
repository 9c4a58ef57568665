// extern "C" entry points of libtemf_b200 (declared in include/temf_b200.h).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>

#include "../../include/temf_b200.h"
#include "adjoint.h"
#include "assemble.h"
#include "batch.h"
#include "factor.h"
#include "fetd.h"
#include "solve.h"

using namespace temf;

struct temf_run_state {
  RunResult res;
  bool valid = false;
};

struct temf_batch {
  temf::Batch b;
  std::string err;
};

namespace {

// per-context extras that do not belong in the core context header
struct CtxExtra {
  temf_run_state run;
  AdjointResult adj;
  bool adj_valid = false;
  // PARDISO shim: user upper-CSR position -> CSR position of the permuted full pattern
  std::vector<int> shim_map;  // nnz_user (index into pattern) or -1
  std::vector<int> shim_map_up;  // the mirrored (upper) position of each off-diagonal entry, -1 on the diagonal
  int shim_n = 0, shim_nnz = 0;
  int shim_max = 0;
  DBuf<double> shim_vals;     // user values on device
  DBuf<int> shim_map_d, shim_map_up_d;
  DBuf<double> vec;           // scratch vectors for host-facing solves
  DBuf<double*> lb;           // device word holding the factor base for host solves
  DBuf<double> shim_full[2];  // PARDISO shim: the user's matrix of each slot on the permuted pattern
  DBuf<int> perm;             // fill-reducing permutation on the device (perm[new] = old)
};

// Contexts may live on different host threads: the registry is locked.  An
// entry is created on first use and freed by temf_destroy (drop_extra), so a
// new context at a reused address starts from a fresh entry.
std::mutex& registry_lock() {
  static std::mutex m;
  return m;
}
std::vector<std::pair<temf_ctx*, CtxExtra*>>& registry() {
  static std::vector<std::pair<temf_ctx*, CtxExtra*>> r;
  return r;
}
CtxExtra& extra(temf_ctx* c) {
  std::lock_guard<std::mutex> g(registry_lock());
  for (auto& p : registry())
    if (p.first == c) return *p.second;
  registry().push_back({c, new CtxExtra()});
  return *registry().back().second;
}
void drop_extra(temf_ctx* c) {
  std::lock_guard<std::mutex> g(registry_lock());
  auto& r = registry();
  for (size_t i = 0; i < r.size(); ++i)
    if (r[i].first == c) { delete r[i].second; r.erase(r.begin() + i); return; }
}

template <typename F>
int guarded(temf_ctx* c, F&& f) {
  if (!c) return TEMF_EARG;
  try {
    if (c->device >= 0) {
      cudaError_t e = cudaSetDevice(c->device);
      if (e != cudaSuccess) throw CudaError(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
    c->err.clear();
    return f();
  } catch (const ArgError& e) {
    c->err = e.what();
    return TEMF_EARG;
  } catch (const StateError& e) {
    c->err = e.what();
    return TEMF_ESTATE;
  } catch (const CudaError& e) {
    c->err = e.what();
    return TEMF_ECUDA;
  } catch (const std::exception& e) {
    c->err = e.what();
    return TEMF_EINTERNAL;
  }
}

template <typename F>
int guarded_batch(temf_batch* B, F&& f) {
  if (!B) return TEMF_EARG;
  try {
    TEMF_CUDA(cudaSetDevice(B->b.device));
    B->err.clear();
    return f();
  } catch (const ArgError& e) {
    B->err = e.what();
    return TEMF_EARG;
  } catch (const StateError& e) {
    B->err = e.what();
    return TEMF_ESTATE;
  } catch (const CudaError& e) {
    B->err = e.what();
    return TEMF_ECUDA;
  } catch (const std::exception& e) {
    B->err = e.what();
    return TEMF_EINTERNAL;
  }
}


// K7 set-up: n_arr / d_arr (src/FETD_FWD.f90:712-731) for each receiver.
// lambda'_k = a_k + b_k x + c_k y + d_k z is evaluated as six times the signed
// volume of the tet with vertex k replaced by the receiver point.
__global__ void k_receiver_operators(int nrec, const double* __restrict__ xyz, const int* __restrict__ tet_vex,
                                     const int* __restrict__ tet_drc, const int* __restrict__ rec_tet,
                                     const double* __restrict__ rec_cor, double* __restrict__ w) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrec) return;
  const int t = rec_tet[r];
  double X[4][3];
  for (int k = 0; k < 4; ++k)
    for (int a = 0; a < 3; ++a) X[k][a] = xyz[3 * (int64_t)tet_vex[4 * (int64_t)t + k] + a];
  const double P[3] = {rec_cor[3 * r], rec_cor[3 * r + 1], rec_cor[3 * r + 2]};
  auto vol6 = [](const double A[4][3]) {
    const double ax = A[1][0] - A[0][0], ay = A[1][1] - A[0][1], az = A[1][2] - A[0][2];
    const double bx = A[2][0] - A[0][0], by = A[2][1] - A[0][1], bz = A[2][2] - A[0][2];
    const double cx = A[3][0] - A[0][0], cy = A[3][1] - A[0][1], cz = A[3][2] - A[0][2];
    return ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
  };
  const double v6 = vol6(X);
  double lam[4];
  for (int k = 0; k < 4; ++k) {
    double Y[4][3];
    for (int m = 0; m < 4; ++m)
      for (int a = 0; a < 3; ++a) Y[m][a] = (m == k) ? P[a] : X[m][a];
    lam[k] = vol6(Y);
  }
  // gradients (b,c,d) as in the assembly kernel
  auto D = [&](int u, int wv, int p, int q, int rr) {
    return (X[q][u] - X[p][u]) * (X[rr][wv] - X[p][wv]) - (X[rr][u] - X[p][u]) * (X[q][wv] - X[p][wv]);
  };
  const int rest[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  const double sa[4] = {1.0, -1.0, 1.0, -1.0};
  double g[4][3];
  for (int k = 0; k < 4; ++k) {
    const int p = rest[k][0], q = rest[k][1], rr = rest[k][2];
    g[k][0] = -sa[k] * D(1, 2, p, q, rr);
    g[k][1] = sa[k] * D(0, 2, p, q, rr);
    g[k][2] = -sa[k] * D(0, 1, p, q, rr);
  }
  const int it[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {3, 1}, {2, 3}};
  for (int j = 0; j < 6; ++j) {
    const int p = it[j][0], q = it[j][1];
    const double dx = X[p][0] - X[q][0], dy = X[p][1] - X[q][1], dz = X[p][2] - X[q][2];
    const double len = sqrt(dx * dx + dy * dy + dz * dz);
    const double sc = len / (v6 * v6);
    const double s = (double)tet_drc[6 * (int64_t)t + j];
    double nv[3], dv[3];
    for (int a = 0; a < 3; ++a) nv[a] = (lam[p] * g[q][a] - lam[q] * g[p][a]) * sc;
    dv[0] = -2.0 * (g[p][1] * g[q][2] - g[q][1] * g[p][2]) * sc;
    dv[1] = -2.0 * (g[q][0] * g[p][2] - g[p][0] * g[q][2]) * sc;
    dv[2] = -2.0 * (g[p][0] * g[q][1] - g[q][0] * g[p][1]) * sc;
    for (int a = 0; a < 3; ++a) {
      w[r * 36 + a * 6 + j] = nv[a] * s;
      w[r * 36 + (3 + a) * 6 + j] = dv[a] * s;
    }
  }
}

// p_in_tet (src/FETD_FWD.f90:1009-1049): first tet in order whose centroid is
// within rec_charac and whose five determinants share a sign.  One warp per point.
__global__ void k_locate(int npts, const double* __restrict__ pts, double rc, int n_tets,
                         const double* __restrict__ xyz, const int* __restrict__ tet_vex, int* __restrict__ out) {
  const int pt = blockIdx.x;
  if (pt >= npts) return;
  const double p[3] = {pts[3 * pt], pts[3 * pt + 1], pts[3 * pt + 2]};
  __shared__ int best;
  if (threadIdx.x == 0) best = INT_MAX;
  __syncthreads();
  auto det4 = [](const double A[4][3]) {  // det [[x y z 1]] rows
    const double ax = A[1][0] - A[0][0], ay = A[1][1] - A[0][1], az = A[1][2] - A[0][2];
    const double bx = A[2][0] - A[0][0], by = A[2][1] - A[0][1], bz = A[2][2] - A[0][2];
    const double cx = A[3][0] - A[0][0], cy = A[3][1] - A[0][1], cz = A[3][2] - A[0][2];
    return -(ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx));
  };
  for (int t = threadIdx.x; t < n_tets; t += blockDim.x) {
    if (t >= best) break;
    double X[4][3];
    double m[3] = {0, 0, 0};
    for (int k = 0; k < 4; ++k)
      for (int a = 0; a < 3; ++a) { X[k][a] = xyz[3 * (int64_t)tet_vex[4 * (int64_t)t + k] + a]; m[a] += X[k][a]; }
    const double dx = m[0] / 4.0 - p[0], dy = m[1] / 4.0 - p[1], dz = m[2] / 4.0 - p[2];
    if (sqrt(dx * dx + dy * dy + dz * dz) > rc) continue;
    double d[5];
    d[0] = det4(X);
    for (int k = 0; k < 4; ++k) {
      double Y[4][3];
      for (int q = 0; q < 4; ++q)
        for (int a = 0; a < 3; ++a) Y[q][a] = (q == k) ? p[a] : X[q][a];
      d[k + 1] = det4(Y);
    }
    bool pos = true, neg = true;
    for (int k = 0; k < 5; ++k) { pos &= d[k] >= 0.0; neg &= d[k] <= 0.0; }
    if (pos || neg) atomicMin(&best, t);
  }
  __syncthreads();
  if (threadIdx.x == 0) out[pt] = best == INT_MAX ? 0 : best + 1;
}

__global__ void k_scatter_user(int64_t nnz, const int* __restrict__ map, const double* __restrict__ va,
                               double* __restrict__ dst) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < nnz && map[q] >= 0) dst[map[q]] = va[q];
}

__global__ void k_permute_in(int n, int nrhs, const int* __restrict__ perm, const double* __restrict__ src,
                             int64_t ld, double* __restrict__ dst) {
  // dst[new*nrhs + c] = src[c*ld + perm[new]]
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)n * nrhs) return;
  const int i = (int)(gid / nrhs), c = (int)(gid % nrhs);
  dst[gid] = src[(int64_t)c * ld + perm[i]];
}
__global__ void k_permute_out(int n, int nrhs, const int* __restrict__ perm, const double* __restrict__ src,
                              int64_t ld, double* __restrict__ dst) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)n * nrhs) return;
  const int i = (int)(gid / nrhs), c = (int)(gid % nrhs);
  dst[(int64_t)c * ld + perm[i]] = src[gid];
}

DBuf<int>& perm_dev(temf_ctx* c) { return extra(c).perm; }

}  // namespace

namespace temf {
// Device copy of the fill-reducing permutation (perm[new] = old) of a context.
const int* ctx_perm_device(temf_ctx* c) { return perm_dev(c).p; }
}  // namespace temf

namespace {

void need(bool cond, const char* msg) {
  if (!cond) throw StateError(msg);
}

}  // namespace

namespace {

// Edge keys of every (tet, local edge) of a 1-based tet_vex(n_tets, 4)
// (column-major): key = min vertex << bits | max vertex, local edges joining
// the vertex pairs ind_tet (src/FETD_FWD.f90:23), sorted ascending: a
// counting sort by the smaller vertex, then an insertion sort by the larger
// one inside each (short) bucket.  Both are stable, so equal keys stay in
// (tet, local edge) order.  slot[p] = 6 * tet + local edge of the p-th key.
struct EdgeKeys {
  std::vector<uint64_t> key;
  std::vector<int64_t> slot;
  int bits = 0;
};

bool edge_keys(int n_tets, const int* tet_vex, EdgeKeys& K) {
  static const int it[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {3, 1}, {2, 3}};
  const int64_t m = 6LL * n_tets;
  int64_t vmax = 0;
  for (int64_t q = 0; q < 4LL * n_tets; ++q) {
    if (tet_vex[q] < 0) return false;
    vmax = std::max<int64_t>(vmax, tet_vex[q]);
  }
  int bits = 1;
  while ((1LL << bits) <= vmax) ++bits;
  K.bits = bits;
  auto lo_hi = [&](int64_t q, uint64_t& a, uint64_t& b) {
    const int64_t t = q / 6, j = q % 6;
    a = (uint64_t)tet_vex[it[j][0] * (int64_t)n_tets + t];
    b = (uint64_t)tet_vex[it[j][1] * (int64_t)n_tets + t];
    if (a > b) std::swap(a, b);
  };
  std::vector<int64_t> start(vmax + 2, 0);
  for (int64_t q = 0; q < m; ++q) {
    uint64_t a, b;
    lo_hi(q, a, b);
    ++start[a + 1];
  }
  for (int64_t v = 0; v <= vmax; ++v) start[v + 1] += start[v];
  K.key.resize(m);
  K.slot.resize(m);
  {
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (int64_t q = 0; q < m; ++q) {
      uint64_t a, b;
      lo_hi(q, a, b);
      const int64_t d = fill[a]++;
      K.key[d] = (a << bits) | b;
      K.slot[d] = q;
    }
  }
  for (int64_t v = 0; v <= vmax; ++v)
    for (int64_t p = start[v] + 1; p < start[v + 1]; ++p) {
      const uint64_t k = K.key[p];
      const int64_t sl = K.slot[p];
      int64_t r = p;
      for (; r > start[v] && K.key[r - 1] > k; --r) {
        K.key[r] = K.key[r - 1];
        K.slot[r] = K.slot[r - 1];
      }
      K.key[r] = k;
      K.slot[r] = sl;
    }
  return true;
}

}  // namespace

extern "C" {

const char* temf_version(void) { return "temf_b200 0.1 (sm_100a, FP64)"; }

int temf_create(int device, temf_ctx** out) {
  if (!out) return TEMF_EARG;
  *out = nullptr;
  temf_ctx* c = new temf_ctx();
  c->device = device;
  int rc = guarded(c, [&] {
    TEMF_CUDA(cudaSetDevice(device));
    TEMF_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->d_status.alloc(4);
    TEMF_CUDA(cudaMemset(c->d_status.p, 0, 4 * sizeof(int)));
    return TEMF_OK;
  });
  if (rc != TEMF_OK) {
    // keep the context so the caller can read the message
    *out = c;
    return rc;
  }
  *out = c;
  return TEMF_OK;
}

int temf_destroy(temf_ctx* c) {
  if (!c) return TEMF_EARG;
  if (c->device >= 0) cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  drop_extra(c);
  cudaStream_t s = c->stream;
  delete c;
  if (s) cudaStreamDestroy(s);
  return TEMF_OK;
}

const char* temf_last_error(const temf_ctx* c) { return c ? c->err.c_str() : "null context"; }

int temf_mesh_count_edges(int n_tets, const int* tet_vex, int* n_edges) {
  if (n_tets <= 0 || !tet_vex || !n_edges) return TEMF_EARG;
  try {
    EdgeKeys K;
    if (!edge_keys(n_tets, tet_vex, K)) return TEMF_EARG;
    int64_t count = 0;
    for (size_t p = 0; p < K.key.size(); ++p)
      if (p == 0 || K.key[p] != K.key[p - 1]) ++count;
    if (count > INT32_MAX) return TEMF_EARG;
    *n_edges = (int)count;
    return TEMF_OK;
  } catch (...) {
    return TEMF_EINTERNAL;
  }
}

int temf_mesh_topology(int n_tets, const int* tet_vex, int n_edges, int* edg_vex, int* tet_edg, int* tet_drc) {
  if (n_tets <= 0 || !tet_vex || !edg_vex || !tet_edg || !tet_drc) return TEMF_EARG;
  try {
    EdgeKeys K;
    if (!edge_keys(n_tets, tet_vex, K)) return TEMF_EARG;
    int64_t count = 0;
    for (size_t p = 0; p < K.key.size(); ++p)
      if (p == 0 || K.key[p] != K.key[p - 1]) ++count;
    if (count != n_edges) return TEMF_EARG;
    // edges in ascending (min, max) order; every (tet, local edge) gets its edge's 1-based index
    int64_t e = -1;
    for (size_t p = 0; p < K.key.size(); ++p) {
      if (p == 0 || K.key[p] != K.key[p - 1]) {
        ++e;
        edg_vex[e] = (int)(K.key[p] >> K.bits);
        edg_vex[(int64_t)n_edges + e] = (int)(K.key[p] & ((1ULL << K.bits) - 1));
      }
      const int64_t q = K.slot[p], t = q / 6, j = q % 6;
      tet_edg[j * n_tets + t] = (int)e + 1;
    }
    static const int it[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {3, 1}, {2, 3}};
    for (int t = 0; t < n_tets; ++t)
      for (int j = 0; j < 6; ++j) {
        const int a = tet_vex[(int64_t)it[j][0] * n_tets + t], b = tet_vex[(int64_t)it[j][1] * n_tets + t];
        tet_drc[(int64_t)j * n_tets + t] = a < b ? 1 : -1;
      }
    return TEMF_OK;
  } catch (...) {
    return TEMF_EINTERNAL;
  }
}

int temf_set_mesh(temf_ctx* c, int n_nodes, const double* nod_cor, int n_tets, const int* tet_vex, int n_edges,
                  const int* edg_vex, const int* tet_edg, const int* tet_drc) {
  return guarded(c, [&] {
    if (n_nodes <= 0 || n_tets <= 0 || n_edges <= 0 || !nod_cor || !tet_vex || !edg_vex || !tet_edg || !tet_drc)
      throw ArgError("temf_set_mesh: empty mesh or NULL array");
    c->n_nodes = n_nodes;
    c->n_tets = n_tets;
    c->n_edges = n_edges;
    c->xyz.resize(3LL * n_nodes);
    for (int i = 0; i < n_nodes; ++i)
      for (int a = 0; a < 3; ++a) c->xyz[3LL * i + a] = nod_cor[(int64_t)a * n_nodes + i];
    c->tet_vex.resize(4LL * n_tets);
    c->tet_edg.resize(6LL * n_tets);
    c->tet_drc.resize(6LL * n_tets);
    for (int t = 0; t < n_tets; ++t) {
      for (int k = 0; k < 4; ++k) {
        const int v = tet_vex[(int64_t)k * n_tets + t];
        if (v < 1 || v > n_nodes) throw ArgError("tet_vex out of range (1-based vertex expected)");
        c->tet_vex[4LL * t + k] = v - 1;
      }
      for (int j = 0; j < 6; ++j) {
        const int e = tet_edg[(int64_t)j * n_tets + t];
        const int d = tet_drc[(int64_t)j * n_tets + t];
        if (e < 1 || e > n_edges) throw ArgError("tet_edg out of range (1-based edge expected)");
        if (d != 1 && d != -1) throw ArgError("tet_drc must be +1 or -1");
        c->tet_edg[6LL * t + j] = e - 1;
        c->tet_drc[6LL * t + j] = d;
      }
    }
    c->edg_vex.resize(2LL * n_edges);
    for (int e = 0; e < n_edges; ++e)
      for (int k = 0; k < 2; ++k) {
        const int v = edg_vex[(int64_t)k * n_edges + e];
        if (v < 1 || v > n_nodes) throw ArgError("edg_vex out of range");
        c->edg_vex[2LL * e + k] = v - 1;
      }
    c->have_mesh = true;
    c->analysed = false;
    c->assembled = false;
    c->slots[0].valid = c->slots[1].valid = false;
    upload_mesh(*c);
    TEMF_CUDA(cudaStreamSynchronize(c->stream));
    return TEMF_OK;
  });
}

int temf_set_media(temf_ctx* c, const double* sig, const double* mu) {
  return guarded(c, [&] {
    need(c->have_mesh, "temf_set_media: set the mesh first");
    if (!sig || !mu) throw ArgError("temf_set_media: NULL array");
    c->aniso = false;
    c->sig.assign(sig, sig + c->n_tets);
    c->mu.assign(mu, mu + c->n_tets);
    for (int t = 0; t < c->n_tets; ++t)
      if (!(c->sig[t] >= 0.0) || !(c->mu[t] > 0.0)) throw ArgError("sigma must be >= 0 and mu > 0 in every tet");
    c->have_media = true;
    c->assembled = false;
    c->adj.valid = false;
    c->slots[0].valid = c->slots[1].valid = false;
    upload_media(*c);
    TEMF_CUDA(cudaStreamSynchronize(c->stream));
    return TEMF_OK;
  });
}

int temf_set_media_tensor(temf_ctx* c, const double* sig9, const double* mu9) {
  return guarded(c, [&] {
    need(c->have_mesh, "temf_set_media_tensor: set the mesh first");
    if (!sig9 || !mu9) throw ArgError("temf_set_media_tensor: NULL array");
    const size_t m = 9 * (size_t)c->n_tets;
    c->sig9.assign(sig9, sig9 + m);
    c->tm9.resize(m);
    for (size_t q = 0; q < m; ++q) {
      if (!std::isfinite(sig9[q]) || !std::isfinite(mu9[q])) throw ArgError("media tensors must be finite");
      c->tm9[q] = mu9[q] == 0.0 ? 0.0 : 1.0 / mu9[q];  // mesh_process's elementwise reciprocal (:624-633)
    }
    // scalar summaries (trace / 3) for the callers that read sigma per tet
    c->sig.assign(c->n_tets, 0.0);
    c->mu.assign(c->n_tets, 0.0);
    for (int t = 0; t < c->n_tets; ++t) {
      c->sig[t] = (sig9[9LL * t] + sig9[9LL * t + 4] + sig9[9LL * t + 8]) / 3.0;
      c->mu[t] = (mu9[9LL * t] + mu9[9LL * t + 4] + mu9[9LL * t + 8]) / 3.0;
    }
    c->aniso = true;
    c->have_media = true;
    c->assembled = false;
    c->adj.valid = false;
    c->slots[0].valid = c->slots[1].valid = false;
    upload_media(*c);
    TEMF_CUDA(cudaStreamSynchronize(c->stream));
    return TEMF_OK;
  });
}

int temf_set_boundary(temf_ctx* c, int bound_cond, const unsigned char* face_mask) {
  return guarded(c, [&] {
    need(c->have_mesh, "temf_set_boundary: set the mesh first");
    if (bound_cond != 0 && bound_cond != 1) throw ArgError("boundary condition must be 0 (PEC) or 1 (first-order ABC)");
    c->bound_cond = bound_cond;
    if (bound_cond) {
      if (face_mask) c->face_mask.assign(face_mask, face_mask + c->n_tets);
      else boundary_face_mask(*c, c->face_mask);
      for (unsigned char v : c->face_mask)
        if (v > 15) throw ArgError("face mask: 4 bits per tet");
      c->d_face_mask.upload(c->face_mask.data(), c->face_mask.size(), c->stream);
      TEMF_CUDA(cudaStreamSynchronize(c->stream));
    }
    c->assembled = false;
    c->adj.valid = false;
    c->slots[0].valid = c->slots[1].valid = false;
    return TEMF_OK;
  });
}

int temf_analyse(temf_ctx* c) {
  return guarded(c, [&] {
    need(c->have_mesh, "temf_analyse: set the mesh first");
    std::vector<int64_t> xadj;
    std::vector<int> adj;
    build_adjacency(*c, xadj, adj);
    // adjacency without the diagonal, edge midpoints as coordinates
    std::vector<int64_t> x2(c->n_edges + 1, 0);
    std::vector<int> a2;
    a2.reserve(adj.size());
    for (int e = 0; e < c->n_edges; ++e) {
      for (int64_t p = xadj[e]; p < xadj[e + 1]; ++p)
        if (adj[p] != e) a2.push_back(adj[p]);
      x2[e + 1] = (int64_t)a2.size();
    }
    std::vector<double> mid(3LL * c->n_edges);
    for (int e = 0; e < c->n_edges; ++e)
      for (int a = 0; a < 3; ++a)
        mid[3LL * e + a] = 0.5 * (c->xyz[3LL * c->edg_vex[2LL * e] + a] + c->xyz[3LL * c->edg_vex[2LL * e + 1] + a]);
    c->sym_opt.max_sn_cols = kSnCols;
    // a new ordering invalidates the mesh-field plan's permuted edges
    c->mf.times.clear();
    c->mf.done.clear();
    c->mf.edges.reset();
    c->mf.b.reset();
    c->mf.snap.reset();
    analyse(c->n_edges, x2.data(), a2.data(), mid.data(), c->sym_opt, c->sym);
    build_pattern(*c, c->sym.perm, c->sym.iperm, c->pat);
    upload_pattern(*c);
    build_factor_plan(*c);
    build_solve_plan(*c);
    perm_dev(c).upload(c->sym.perm.data(), c->sym.perm.size(), c->stream);
    TEMF_CUDA(cudaStreamSynchronize(c->stream));
    c->analysed = true;
    c->assembled = false;
    c->slots[0].valid = c->slots[1].valid = false;
    return TEMF_OK;
  });
}

int temf_assemble(temf_ctx* c) {
  return guarded(c, [&] {
    need(c->analysed, "temf_assemble: call temf_analyse first");
    need(c->have_media, "temf_assemble: set the media first");
    launch_assembly(*c);
    TEMF_CUDA(cudaStreamSynchronize(c->stream));
    c->assembled = true;
    c->slots[0].valid = c->slots[1].valid = false;
    return TEMF_OK;
  });
}

int temf_get_matrix(temf_ctx* c, int which, int* nnz_out, int* ia, int* ja, double* va) {
  return guarded(c, [&] {
    need(c->assembled, "temf_get_matrix: assemble first");
    if (which != 0 && which != 1) throw ArgError("which must be 0 (M_sigma) or 1 (K)");
    const Pattern& P = c->pat;
    const int n = P.n;
    int64_t cnt = 0;
    for (int r = 0; r < n; ++r)
      for (int p = P.rowptr[r]; p < P.rowptr[r + 1]; ++p)
        if (c->sym.perm[P.col[p]] >= c->sym.perm[r]) ++cnt;
    if (nnz_out) *nnz_out = (int)cnt;
    if (!ia && !ja && !va) return TEMF_OK;
    if (!ia || !ja || !va) throw ArgError("ia, ja and va must all be given");
    std::vector<double> vals(P.nnz);
    TEMF_CUDA(cudaMemcpy(vals.data(), which == 0 ? c->d_M.p : c->d_K.p, P.nnz * sizeof(double),
                         cudaMemcpyDeviceToHost));
    std::vector<std::vector<std::pair<int, double>>> rows(n);
    for (int r = 0; r < n; ++r) {
      const int i = c->sym.perm[r];
      for (int p = P.rowptr[r]; p < P.rowptr[r + 1]; ++p) {
        const int j = c->sym.perm[P.col[p]];
        if (j >= i) rows[i].push_back({j, vals[p]});
      }
    }
    int64_t q = 0;
    ia[0] = 1;
    for (int i = 0; i < n; ++i) {
      std::sort(rows[i].begin(), rows[i].end());
      for (auto& e : rows[i]) { ja[q] = e.first + 1; va[q] = e.second; ++q; }
      ia[i + 1] = (int)q + 1;
    }
    return TEMF_OK;
  });
}

int temf_factor(temf_ctx* c, int slot, double dt) {
  return guarded(c, [&] {
    need(c->assembled, "temf_factor: assemble first");
    if (slot != 1 && slot != 2) throw ArgError("slot must be 1 or 2");
    if (!(dt > 0.0)) throw ArgError("dt must be positive");
    return numeric_factor_values_fallback(*c, slot - 1, c->d_M.p, 3.0, c->d_K.p, 2.0 * dt);
  });
}

int temf_release(temf_ctx* c, int slot) {
  return guarded(c, [&] {
    if (slot != 1 && slot != 2) throw ArgError("slot must be 1 or 2");
    c->slots[slot - 1].valid = false;
    return TEMF_OK;
  });
}

__global__ void k_axpy(int64_t n, const double* __restrict__ d, double* __restrict__ x) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) x[q] += d[q];
}

// Iterative refinement steps after a solve with an indefinite factor (the
// reference's PARDISO runs two by default when pivots were perturbed).
constexpr int kRefineSteps = 2;

static void host_solve(temf_ctx* c, int slot0, int nrhs, const double* b, double* x, int ld) {
  CtxExtra& X = extra(c);
  const int n = c->n_edges;
  const size_t vec = (size_t)n * nrhs;
  const FactorSlot& fs = c->slots[slot0];
  const bool refine = fs.indefinite;
  if (X.vec.n < (refine ? 4 : 2) * vec) X.vec.alloc((refine ? 4 : 2) * vec);
  double* dcol = X.vec.p;        // column-major staging
  double* drow = X.vec.p + vec;  // permuted row-major
  cudaStream_t st = c->stream;
  for (int q = 0; q < nrhs; ++q)
    TEMF_CUDA(cudaMemcpyAsync(dcol + (size_t)q * n, b + (size_t)q * ld, n * sizeof(double), cudaMemcpyHostToDevice, st));
  k_permute_in<<<ceil_div((int64_t)vec, 256), 256, 0, st>>>(n, nrhs, perm_dev(c).p, dcol, n, drow);
  TEMF_CHECK_LAUNCH();
  if (!X.lb.p) X.lb.alloc(1);
  double* Lp = fs.L.p;
  TEMF_CUDA(cudaMemcpyAsync(X.lb.p, &Lp, sizeof(double*), cudaMemcpyHostToDevice, st));
  const double* sgn = fs.indefinite ? fs.sgn.p : nullptr;
  if (refine) {
    // x = A^-1 b, then x += A^-1 (b - A x), kRefineSteps times
    double* bp = X.vec.p + 2 * vec;  // b, permuted
    double* r = X.vec.p + 3 * vec;   // residual, then correction
    TEMF_CUDA(cudaMemcpyAsync(bp, drow, vec * sizeof(double), cudaMemcpyDeviceToDevice, st));
    launch_solve(*c, X.lb.p, drow, nrhs, st, sgn);
    for (int it = 0; it < kRefineSteps; ++it) {
      launch_residual(*c, fs, drow, bp, r, nrhs, st);
      launch_solve(*c, X.lb.p, r, nrhs, st, sgn);
      k_axpy<<<ceil_div((int64_t)vec, 256), 256, 0, st>>>((int64_t)vec, r, drow);
      TEMF_CHECK_LAUNCH();
    }
  } else {
    launch_solve(*c, X.lb.p, drow, nrhs, st);
  }
  k_permute_out<<<ceil_div((int64_t)vec, 256), 256, 0, st>>>(n, nrhs, perm_dev(c).p, drow, n, dcol);
  TEMF_CHECK_LAUNCH();
  for (int q = 0; q < nrhs; ++q)
    TEMF_CUDA(cudaMemcpyAsync(x + (size_t)q * ld, dcol + (size_t)q * n, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  TEMF_CUDA(cudaStreamSynchronize(st));
  if (const int fl = solve_error_flag(*c)) {
    clear_solve_error_flag(*c);
    throw StateError("a triangular-solve wait timed out (code " + std::to_string(fl) + ")");
  }
}

int temf_solve(temf_ctx* c, int slot, int nrhs, const double* b, double* x, int ld) {
  return guarded(c, [&] {
    if (slot != 1 && slot != 2) throw ArgError("slot must be 1 or 2");
    need(c->slots[slot - 1].valid, "temf_solve: the slot holds no valid factor");
    if (nrhs < 1 || ld < c->n_edges || !b || !x) throw ArgError("temf_solve: bad nrhs/ld/pointers");
    host_solve(c, slot - 1, nrhs, b, x, ld);
    return TEMF_OK;
  });
}

int temf_spmv(temf_ctx* c, int which, int nrhs, const double* x, double* y, int ld) {
  return guarded(c, [&] {
    need(c->assembled, "temf_spmv: assemble first");
    if (which != 0 && which != 1) throw ArgError("which must be 0 or 1");
    if (nrhs < 1 || ld < c->n_edges || !x || !y) throw ArgError("temf_spmv: bad arguments");
    CtxExtra& X = extra(c);
    const int n = c->n_edges;
    const size_t vec = (size_t)n * nrhs;
    if (X.vec.n < 3 * vec) X.vec.alloc(3 * vec);
    double *dcol = X.vec.p, *din = X.vec.p + vec, *dout = X.vec.p + 2 * vec;
    cudaStream_t st = c->stream;
    for (int q = 0; q < nrhs; ++q)
      TEMF_CUDA(cudaMemcpyAsync(dcol + (size_t)q * n, x + (size_t)q * ld, n * sizeof(double), cudaMemcpyHostToDevice, st));
    k_permute_in<<<ceil_div((int64_t)vec, 256), 256, 0, st>>>(n, nrhs, perm_dev(c).p, dcol, n, din);
    launch_spmv(*c, which == 0 ? c->d_M.p : c->d_K.p, din, dout, nrhs, st);
    k_permute_out<<<ceil_div((int64_t)vec, 256), 256, 0, st>>>(n, nrhs, perm_dev(c).p, dout, n, dcol);
    TEMF_CHECK_LAUNCH();
    for (int q = 0; q < nrhs; ++q)
      TEMF_CUDA(cudaMemcpyAsync(y + (size_t)q * ld, dcol + (size_t)q * n, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    TEMF_CUDA(cudaStreamSynchronize(st));
    return TEMF_OK;
  });
}

int temf_set_sources(temf_ctx* c, int nrhs, const int* col_ptr, const int* src_edg, const int* src_drc,
                     int source_type, int pulse_type, double t0, double current) {
  return guarded(c, [&] {
    need(c->analysed, "temf_set_sources: call temf_analyse first");
    if (nrhs < 1 || !col_ptr || (col_ptr[nrhs] > 0 && (!src_edg || !src_drc))) throw ArgError("bad source arrays");
    if (source_type != 1 || pulse_type < 1 || pulse_type > 3) throw ArgError("source_type must be 1, pulse_type 1..3");
    if (!(t0 > 0.0)) throw ArgError("pulse width t0 must be positive");
    Source& S = c->src;
    S.nrhs = nrhs;
    S.source_type = source_type;
    S.pulse_type = pulse_type;
    S.t0 = t0;
    S.current = current;
    S.ptr.assign(nrhs + 1, 0);
    S.idx.clear();
    S.rhs_col.clear();
    S.coef.clear();
    for (int q = 0; q < nrhs; ++q) {
      if (col_ptr[q + 1] < col_ptr[q]) throw ArgError("col_ptr must be non-decreasing");
      // last assignment wins (r_h(src_edg(i)) = ..., src/FETD_FWD.f90:1507)
      std::vector<std::pair<int, double>> ent;
      for (int k = col_ptr[q]; k < col_ptr[q + 1]; ++k) {
        const int e = src_edg[k] - 1;
        if (e < 0 || e >= c->n_edges) throw ArgError("src_edg out of range");
        const int a = c->edg_vex[2LL * e], b = c->edg_vex[2LL * e + 1];
        const double dx = c->xyz[3LL * a] - c->xyz[3LL * b], dy = c->xyz[3LL * a + 1] - c->xyz[3LL * b + 1],
                     dz = c->xyz[3LL * a + 2] - c->xyz[3LL * b + 2];
        const double v = (double)src_drc[k] * std::sqrt(dx * dx + dy * dy + dz * dz);
        bool found = false;
        for (auto& p : ent)
          if (p.first == e) { p.second = v; found = true; }
        if (!found) ent.push_back({e, v});
      }
      for (auto& p : ent) {
        S.idx.push_back(c->sym.iperm[p.first]);
        S.rhs_col.push_back(q);
        S.coef.push_back(p.second);
      }
      S.ptr[q + 1] = (int)S.idx.size();
    }
    S.d_idx.upload(S.idx.data(), S.idx.size(), c->stream);
    S.d_col.upload(S.rhs_col.data(), S.rhs_col.size(), c->stream);
    S.d_coef.upload(S.coef.data(), S.coef.size(), c->stream);
    TEMF_CUDA(cudaStreamSynchronize(c->stream));
    return TEMF_OK;
  });
}

int temf_set_receivers(temf_ctx* c, int nrec, const int* rec_tet, const double* rec_cor, const int* rec_rhs) {
  return guarded(c, [&] {
    need(c->analysed, "temf_set_receivers: call temf_analyse first");
    if (nrec < 0 || (nrec > 0 && (!rec_tet || !rec_cor))) throw ArgError("bad receiver arrays");
    Receivers& R = c->rec;
    R.nrec = nrec;
    R.rec_tet.resize(nrec);
    R.rec_rhs.assign(nrec, 0);
    R.xyz.resize(3LL * nrec);
    std::vector<int> edges(6LL * std::max(nrec, 1));
    for (int r = 0; r < nrec; ++r) {
      const int t = rec_tet[r] - 1;
      if (t < 0 || t >= c->n_tets) throw ArgError("rec_tet out of range (1-based tet expected)");
      R.rec_tet[r] = t;
      if (rec_rhs) R.rec_rhs[r] = rec_rhs[r];
      if (R.rec_rhs[r] < 0) throw ArgError("rec_rhs must be >= 0");
      for (int a = 0; a < 3; ++a) R.xyz[3LL * r + a] = rec_cor[(int64_t)a * nrec + r];
      for (int j = 0; j < 6; ++j) edges[6LL * r + j] = c->sym.iperm[c->tet_edg[6LL * t + j]];
    }
    if (!nrec) return TEMF_OK;
    R.d_edges.upload(edges.data(), edges.size(), c->stream);
    R.d_rhs.upload(R.rec_rhs.data(), R.rec_rhs.size(), c->stream);
    DBuf<int> dt;
    dt.upload(R.rec_tet.data(), R.rec_tet.size(), c->stream);
    DBuf<double> dc;
    dc.upload(R.xyz.data(), R.xyz.size(), c->stream);
    R.d_w.alloc(36LL * nrec);
    k_receiver_operators<<<ceil_div(nrec, 64), 64, 0, c->stream>>>(nrec, c->d_xyz.p, c->d_tet_vex.p,
                                                                    c->d_tet_drc.p, dt.p, dc.p, R.d_w.p);
    TEMF_CHECK_LAUNCH();
    R.w_host.resize(36LL * nrec);
    TEMF_CUDA(cudaMemcpyAsync(R.w_host.data(), R.d_w.p, 36LL * nrec * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
    TEMF_CUDA(cudaStreamSynchronize(c->stream));
    return TEMF_OK;
  });
}

int temf_get_receiver_operators(temf_ctx* c, double* n_arr, double* d_arr) {
  return guarded(c, [&] {
    const Receivers& R = c->rec;
    const int nrec = R.nrec;
    for (int r = 0; r < nrec; ++r) {
      const int t = R.rec_tet[r];
      for (int j = 0; j < 6; ++j) {
        const double s = (double)c->tet_drc[6LL * t + j];  // undo the folded orientation sign
        for (int a = 0; a < 3; ++a) {
          if (n_arr) n_arr[(int64_t)a * 6 * nrec + (int64_t)j * nrec + r] = R.w_host[r * 36 + a * 6 + j] * s;
          if (d_arr) d_arr[(int64_t)a * 6 * nrec + (int64_t)j * nrec + r] = R.w_host[r * 36 + (3 + a) * 6 + j] * s;
        }
      }
    }
    return TEMF_OK;
  });
}

int temf_locate_points(temf_ctx* c, int npts, const double* pts, double rec_charac, int* tet_out) {
  return guarded(c, [&] {
    need(c->have_mesh, "temf_locate_points: set the mesh first");
    if (npts < 0 || (npts && (!pts || !tet_out))) throw ArgError("bad arguments");
    if (!npts) return TEMF_OK;
    std::vector<double> p(3LL * npts);
    for (int i = 0; i < npts; ++i)
      for (int a = 0; a < 3; ++a) p[3LL * i + a] = pts[(int64_t)a * npts + i];
    DBuf<double> dp;
    dp.upload(p.data(), p.size(), c->stream);
    DBuf<int> dout;
    dout.alloc(npts);
    k_locate<<<npts, 256, 0, c->stream>>>(npts, dp.p, rec_charac, c->n_tets, c->d_xyz.p, c->d_tet_vex.p, dout.p);
    TEMF_CHECK_LAUNCH();
    TEMF_CUDA(cudaMemcpyAsync(tet_out, dout.p, npts * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    TEMF_CUDA(cudaStreamSynchronize(c->stream));
    return TEMF_OK;
  });
}

int temf_set_mesh_fields(temf_ctx* c, int n_times, const double* times) {
  return guarded(c, [&] {
    need(c->analysed, "temf_set_mesh_fields: call temf_analyse first");
    if (n_times < 0 || n_times > 30 || (n_times > 0 && !times)) throw ArgError("0 to 30 vtkout times expected");
    temf::MeshFieldPlan& M = c->mf;
    M.times.assign(times, times + n_times);
    M.done.assign(n_times, 0);
    if (n_times == 0) {
      M.edges.reset();
      M.b.reset();
      M.snap.reset();
      return TEMF_OK;
    }
    const int T = c->n_tets;
    std::vector<int> e(6LL * T);
    for (int64_t q = 0; q < 6LL * T; ++q) e[q] = c->sym.iperm[c->tet_edg[q]];
    M.edges.upload(e.data(), e.size(), c->stream);
    M.b.alloc(3LL * T);
    M.snap.alloc(9LL * T * n_times);
    TEMF_CUDA(cudaMemsetAsync(M.snap.p, 0, M.snap.bytes(), c->stream));
    TEMF_CUDA(cudaStreamSynchronize(c->stream));
    return TEMF_OK;
  });
}

int temf_result_mesh_fields(temf_ctx* c, int index, double* fields, int* done) {
  return guarded(c, [&] {
    const temf::MeshFieldPlan& M = c->mf;
    if (index < 0 || index >= M.n()) throw ArgError("no such vtkout time");
    if (done) *done = M.done.size() > (size_t)index ? M.done[index] : 0;
    if (fields) {
      const size_t cnt = 9ULL * c->n_tets;
      TEMF_CUDA(cudaMemcpyAsync(fields, M.snap.p + cnt * index, cnt * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
      TEMF_CUDA(cudaStreamSynchronize(c->stream));
    }
    return TEMF_OK;
  });
}

int temf_run(temf_ctx* c, int sp_division, int sp_double, int sp_dblesize, double time_maximum, int flags,
             const int* forced, int n_forced, int max_steps) {
  return guarded(c, [&] {
    need(c->assembled, "temf_run: assemble first");
    need(c->src.nrhs >= 1, "temf_run: set the sources first");
    for (int r = 0; r < c->rec.nrec; ++r)
      if (c->rec.rec_rhs[r] >= c->src.nrhs) throw ArgError("a receiver samples a RHS column that does not exist");
    RunOptions o;
    o.step_dvsi = sp_division;
    o.step_dble = sp_double;
    o.step_dblesize = sp_dblesize;
    o.time_maximum = time_maximum;
    o.legacy_linux = flags & 1;
    o.use_graphs = (flags & 2) ? 0 : 1;
    o.forced = forced;
    o.n_forced = forced ? n_forced : 0;
    o.max_steps = max_steps;
    o.record_every = c->adj.every;
    CtxExtra& X = extra(c);
    X.run.valid = false;
    c->adj.valid = false;
    run_fetd(*c, o, X.run.res);
    X.run.valid = true;
    c->slots[0].valid = c->slots[1].valid = false;  // the run reused both slots
    return TEMF_OK;
  });
}

int temf_result_rows(temf_ctx* c, int* rows) {
  return guarded(c, [&] {
    CtxExtra& X = extra(c);
    need(X.run.valid, "no completed run");
    if (!rows) throw ArgError("NULL");
    *rows = (int)X.run.res.steps.size();
    return TEMF_OK;
  });
}

// 9 output components per receiver and row (solution_output, src/FETD_FWD.f90:1530-1622)
static void fields_of(temf_ctx* c, std::vector<double>& f) {
  const RunResult& R = extra(c).run.res;
  const int rows = (int)R.steps.size(), nrec = c->rec.nrec;
  f.assign((size_t)rows * nrec * 9, 0.0);
  for (int i = 0; i < rows; ++i)
    for (int r = 0; r < nrec; ++r) {
      const double* s = R.samples.data() + ((size_t)i * nrec + r) * 6;
      double* o = f.data() + ((size_t)i * nrec + r) * 9;
      for (int a = 0; a < 3; ++a) o[a] = s[a];
      for (int a = 0; a < 3; ++a) o[3 + a] = (R.steps[i] == 0) ? 0.0 : s[3 + a];
      for (int a = 0; a < 3; ++a)
        o[6 + a] = (i == 0 ? 0.0 : f[((size_t)(i - 1) * nrec + r) * 9 + 6 + a]) + o[3 + a] * R.dts[i];
    }
}

int temf_result_get(temf_ctx* c, int* step, double* time, double* dt, double* fields) {
  return guarded(c, [&] {
    CtxExtra& X = extra(c);
    need(X.run.valid, "no completed run");
    const RunResult& R = X.run.res;
    const size_t rows = R.steps.size();
    if (step) std::copy(R.steps.begin(), R.steps.end(), step);
    if (time) std::copy(R.times.begin(), R.times.end(), time);
    if (dt) std::copy(R.dts.begin(), R.dts.end(), dt);
    if (fields && rows) {
      std::vector<double> f;
      fields_of(c, f);
      std::copy(f.begin(), f.end(), fields);
    }
    return TEMF_OK;
  });
}

int temf_result_trials(temf_ctx* c, int* n_trials, double* errors, int* accepted) {
  return guarded(c, [&] {
    CtxExtra& X = extra(c);
    need(X.run.valid, "no completed run");
    const RunResult& R = X.run.res;
    if (n_trials) *n_trials = (int)R.trial_err.size();
    if (errors) std::copy(R.trial_err.begin(), R.trial_err.end(), errors);
    if (accepted) std::copy(R.trial_acc.begin(), R.trial_acc.end(), accepted);
    return TEMF_OK;
  });
}

int temf_result_gates(temf_ctx* c, int n_gates, const double* gates, double* out, int* done) {
  return guarded(c, [&] {
    CtxExtra& X = extra(c);
    need(X.run.valid, "no completed run");
    if (n_gates < 0 || (n_gates && (!gates || !out))) throw ArgError("bad arguments");
    const RunResult& R = X.run.res;
    const int rows = (int)R.steps.size(), nrec = c->rec.nrec;
    std::vector<double> f;
    fields_of(c, f);
    const size_t w = (size_t)nrec * 9;
    std::vector<char> ok(n_gates, 0);
    std::fill(out, out + (size_t)n_gates * w, 0.0);
    for (int i = 0; i < rows; ++i) {
      const double t = R.times[i];
      for (int g = 0; g < n_gates; ++g) {
        if (t >= gates[g] && !ok[g]) {
          if (i == 0) {  // the reference copies row 1 and leaves the gate open (exit)
            std::copy(f.begin(), f.begin() + w, out + (size_t)g * w);
            break;
          }
          const double t1 = R.times[i - 1], t2 = t;
          for (size_t k = 0; k < w; ++k) {
            const double y1 = f[(size_t)(i - 1) * w + k], y2 = f[(size_t)i * w + k];
            const double a = (y1 - y2) / (t1 - t2);  // interp_lin, src/FETD_UTILITY.f90:21-31
            const double b = y1 - a * t1;
            out[(size_t)g * w + k] = a * gates[g] + b;
          }
          ok[g] = 1;
        }
      }
    }
    if (done)
      for (int g = 0; g < n_gates; ++g) done[g] = ok[g];
    return TEMF_OK;
  });
}

int temf_result_timing(temf_ctx* c, double* ms_factor, double* ms_steps, double* ms_total, int* n_factor,
                       int* n_solve, long long* n_launch) {
  return guarded(c, [&] {
    CtxExtra& X = extra(c);
    need(X.run.valid, "no completed run");
    const RunResult& R = X.run.res;
    if (ms_factor) *ms_factor = R.ms_factor;
    if (ms_steps) *ms_steps = R.ms_steps;
    if (ms_total) *ms_total = R.ms_total;
    if (n_factor) *n_factor = R.n_factor;
    if (n_solve) *n_solve = R.n_solve;
    if (n_launch) *n_launch = (long long)R.launches;
    return TEMF_OK;
  });
}

// ---- many models at once ---------------------------------------------------
int temf_batch_create(temf_ctx* const* models, int n_models, temf_batch** out) {
  if (!out || !models || n_models < 1) return TEMF_EARG;
  temf_batch* B = new temf_batch();
  *out = B;
  B->b.device = models[0] ? models[0]->device : 0;
  return guarded_batch(B, [&] {
    for (int m = 0; m < n_models; ++m) {
      temf_ctx* c = models[m];
      if (!c) throw ArgError("temf_batch_create: NULL model");
      if (c->device != B->b.device) throw ArgError("temf_batch_create: models on different devices");
      for (int q = 0; q < m; ++q)
        if (models[q] == c) throw ArgError("temf_batch_create: a model appears twice");
      B->b.models.push_back(c);
    }
    TEMF_CUDA(cudaStreamCreateWithFlags(&B->b.stream, cudaStreamNonBlocking));
    return TEMF_OK;
  });
}

int temf_batch_destroy(temf_batch* B) {
  if (!B) return TEMF_EARG;
  cudaSetDevice(B->b.device);
  if (B->b.stream) {
    cudaStreamSynchronize(B->b.stream);
    cudaStreamDestroy(B->b.stream);
  }
  delete B;
  return TEMF_OK;
}

const char* temf_batch_last_error(const temf_batch* B) { return B ? B->err.c_str() : "null batch"; }

int temf_batch_run(temf_batch* B, int sp_division, int sp_double, int sp_dblesize, double time_maximum, int flags,
                   int max_steps) {
  return guarded_batch(B, [&] {
    for (temf_ctx* c : B->b.models) {
      need(c->assembled, "temf_batch_run: assemble every model first");
      need(c->src.nrhs >= 1, "temf_batch_run: set every model's source first");
      for (int r = 0; r < c->rec.nrec; ++r)
        if (c->rec.rec_rhs[r] >= c->src.nrhs) throw ArgError("a receiver samples a RHS column that does not exist");
      if (c->mf.n() > 0) throw ArgError("whole-mesh field dumps are written by temf_run, not by a batch");
      extra(c).run.valid = false;
      c->adj.valid = false;
    }
    RunOptions o;
    o.step_dvsi = sp_division;
    o.step_dble = sp_double;
    o.step_dblesize = sp_dblesize;
    o.time_maximum = time_maximum;
    o.legacy_linux = flags & 1;
    o.use_graphs = (flags & 2) ? 0 : 1;
    o.max_steps = max_steps;
    run_batch(B->b, o, (flags & 4) != 0);
    for (size_t m = 0; m < B->b.models.size(); ++m) {
      CtxExtra& X = extra(B->b.models[m]);
      X.run.res = std::move(B->b.results[m]);
      X.run.valid = true;
    }
    return TEMF_OK;
  });
}

int temf_batch_timing(temf_batch* B, double* ms, long long* counts) {
  return guarded_batch(B, [&] {
    const BatchStats& S = B->b.stats;
    if (ms) { ms[0] = S.ms_total; ms[1] = S.ms_factor; ms[2] = S.ms_steps; ms[3] = S.ms_tune; }
    if (counts) { counts[0] = S.steps; counts[1] = S.launches; counts[2] = S.solves; }
    return TEMF_OK;
  });
}

int temf_batch_tuning(temf_batch* B, int* order, int* grid_pct, double* candidate_ms) {
  return guarded_batch(B, [&] {
    if (order) *order = B->b.tune.order;
    if (grid_pct) *grid_pct = B->b.tune.grid_pct;
    if (candidate_ms)
      for (size_t i = 0; i < B->b.stats.tune_ms.size(); ++i) candidate_ms[i] = B->b.stats.tune_ms[i];
    return B->b.tuned ? 1 : 0;
  });
}

int temf_batch_set_tuning(temf_batch* B, int order, int grid_pct) {
  return guarded_batch(B, [&] {
    if (order < 0 || order > 2 || grid_pct < 1 || grid_pct > 100) throw ArgError("temf_batch_set_tuning: bad value");
    B->b.tune.order = order;
    B->b.tune.grid_pct = grid_pct;
    B->b.tuned = true;
    return TEMF_OK;
  });
}

int temf_tune_solve(temf_ctx* c, int slot, int nrhs, int* split, int* n_cand, int* cand_split, double* cand_ms) {
  return guarded(c, [&] {
    if (slot != 1 && slot != 2) throw ArgError("slot must be 1 or 2");
    if (nrhs < 1) throw ArgError("nrhs must be >= 1");
    need(c->slots[slot - 1].valid, "temf_tune_solve: the slot holds no valid factor");
    clear_solve_error_flag(*c);
    const int best = tune_solve(*c, slot - 1, nrhs);
    if (const int fl = solve_error_flag(*c)) {
      clear_solve_error_flag(*c);
      throw StateError("a triangular-solve wait timed out while tuning (code " + std::to_string(fl) + ")");
    }
    const QueuePlan& Q = nrhs > 1 ? c->splan.qm : c->splan.tree.q;
    if (split) *split = best;
    if (n_cand) *n_cand = (int)Q.tune_ms.size();
    for (size_t i = 0; i < Q.tune_ms.size(); ++i) {
      if (cand_split) cand_split[i] = Q.tune_split[i];
      if (cand_ms) cand_ms[i] = Q.tune_ms[i];
    }
    return TEMF_OK;
  });
}

int temf_solve_schedule(temf_ctx* c, int nrhs, int* split, int* tuned) {
  return guarded(c, [&] {
    need(c->analysed, "temf_solve_schedule: call temf_analyse first");
    const QueuePlan& Q = nrhs > 1 ? c->splan.qm : c->splan.tree.q;
    if (split) *split = Q.split;
    if (tuned) *tuned = Q.tuned ? 1 : 0;
    return TEMF_OK;
  });
}

int temf_set_wait_limit(temf_ctx* c, int spins, int inject_unmet_wait) {
  return guarded(c, [&] {
    if (spins < 0) throw ArgError("temf_set_wait_limit: spins must be >= 0");
    c->spin_limit = spins;
    c->inject_wait = inject_unmet_wait ? 1 : 0;
    return TEMF_OK;
  });
}

int temf_set_solve_plan(temf_ctx* c, int tree_level, int split, int run_leaders) {
  return guarded(c, [&] {
    need(c->analysed, "temf_set_solve_plan: call temf_analyse first");
    set_tree_plan(*c, tree_level, split, run_leaders != 0);
    return TEMF_OK;
  });
}

int temf_solve_plan(temf_ctx* c, int* tree_level, int* split, int* run_leaders, int* n_trees, int* tuned) {
  return guarded(c, [&] {
    need(c->analysed, "temf_solve_plan: call temf_analyse first");
    const TreePlan& T = c->splan.tree;
    if (tree_level) *tree_level = T.level;
    if (split) *split = T.q.split;
    if (run_leaders) *run_leaders = T.leaders ? 1 : 0;
    if (n_trees) *n_trees = T.ntree;
    if (tuned) *tuned = T.tuned ? 1 : 0;
    return TEMF_OK;
  });
}

int temf_solve_timeline(temf_ctx* c, int slot, long long cap, unsigned long long* out, int* n_fwd, int* n_bwd) {
  return guarded(c, [&] {
    if (slot != 1 && slot != 2) throw ArgError("slot must be 1 or 2");
    need(c->slots[slot - 1].valid, "temf_solve_timeline: the slot holds no valid factor");
    if (!n_fwd || !n_bwd) throw ArgError("NULL");
    std::vector<double> ones(c->n_edges, 1.0);
    clear_solve_error_flag(*c);
    solve_timeline(*c, slot - 1, ones.data(), cap, out, n_fwd, n_bwd);
    if (const int fl = solve_error_flag(*c)) {
      clear_solve_error_flag(*c);
      throw StateError("a triangular-solve wait timed out (code " + std::to_string(fl) + ")");
    }
    return TEMF_OK;
  });
}

int temf_adjoint_record(temf_ctx* c, int checkpoint_every) {
  return guarded(c, [&] {
    if (checkpoint_every < 0) throw ArgError("checkpoint_every must be >= 0");
    c->adj.every = checkpoint_every;
    if (!checkpoint_every) {
      c->adj.valid = false;
      c->adj.ck.clear();
    }
    return TEMF_OK;
  });
}

int temf_adjoint(temf_ctx* c, const double* dJ_dfields, int ncell, const int* tet_cell, double* grad_logsigma,
                 double* grad_sigma) {
  return guarded(c, [&] {
    CtxExtra& X = extra(c);
    need(X.run.valid && c->adj.valid, "temf_adjoint: no recorded run (temf_adjoint_record, then temf_run)");
    if (!dJ_dfields) throw ArgError("temf_adjoint: NULL dJ_dfields");
    if (ncell < 0 || (ncell > 0 && grad_logsigma && !tet_cell)) throw ArgError("temf_adjoint: bad cell map");
    const RunResult& R = X.run.res;
    const int rows = (int)R.steps.size(), nrec = c->rec.nrec;
    // fields -> samples: b_i = sum_{m <= i} dB/dt_m dt_m, with dB/dt reported as 0 on step-0 rows
    std::vector<double> g((size_t)rows * nrec * 6, 0.0);
    for (int r = 0; r < nrec; ++r) {
      double tail[3] = {0.0, 0.0, 0.0};
      for (int i = rows - 1; i >= 0; --i) {
        const double* f = dJ_dfields + ((size_t)i * nrec + r) * 9;
        double* o = g.data() + ((size_t)i * nrec + r) * 6;
        for (int a = 0; a < 3; ++a) {
          tail[a] += f[6 + a];
          o[a] = f[a];
          o[3 + a] = (R.steps[i] == 0) ? 0.0 : f[3 + a] + tail[a] * R.dts[i];
        }
      }
    }
    std::vector<int> cell0;
    if (tet_cell) {
      cell0.resize(c->n_tets);
      for (int t = 0; t < c->n_tets; ++t) {
        if (tet_cell[t] < 0 || tet_cell[t] > ncell) throw ArgError("temf_adjoint: tet_cell out of range");
        cell0[t] = tet_cell[t] - 1;
      }
    }
    X.adj_valid = false;
    run_adjoint(*c, g.data(), rows, tet_cell ? cell0.data() : nullptr, ncell, grad_logsigma, grad_sigma, X.adj);
    X.adj_valid = true;
    return TEMF_OK;
  });
}

int temf_adjoint_timing(temf_ctx* c, double* ms, long long* counts) {
  return guarded(c, [&] {
    CtxExtra& X = extra(c);
    need(X.adj_valid, "no completed adjoint sweep");
    if (ms) { ms[0] = X.adj.ms_total; ms[1] = X.adj.ms_factor; }
    if (counts) {
      counts[0] = X.adj.n_nodes;
      counts[1] = X.adj.n_blocks;
      counts[2] = X.adj.n_factor;
      counts[3] = X.adj.launches;
    }
    return TEMF_OK;
  });
}

int temf_set_analysis_options(temf_ctx* c, int leaf_size, int amalg_level) {
  return guarded(c, [&] {
    if (leaf_size < 8 || leaf_size > 100000) throw ArgError("leaf_size must be in [8, 100000]");
    if (amalg_level < 0 || amalg_level > 3) throw ArgError("amalg_level must be 0, 1, 2 or 3");
    c->sym_opt.leaf_size = leaf_size;
    c->sym_opt.amalgamate = amalg_level > 0;
    c->sym_opt.amalg_level = amalg_level;
    return TEMF_OK;
  });
}

int temf_analysis_stats(temf_ctx* c, double* s) {
  return guarded(c, [&] {
    need(c->analysed, "temf_analysis_stats: call temf_analyse first");
    if (!s) throw ArgError("NULL");
    s[0] = c->sym.n;
    s[1] = (double)c->pat.nnz;
    s[2] = c->sym.nsn;
    s[3] = c->sym.nlevels;
    s[4] = (double)c->sym.nnzL;
    s[5] = (double)c->sym.stored;
    s[6] = c->sym.flops;
    s[7] = (double)c->fplan.n_tiles;
    s[8] = c->sym.t_order;
    s[9] = c->sym.t_etree + c->sym.t_colcount + c->sym.t_super;
    return TEMF_OK;
  });
}

int temf_symbolic_host(int n, const long long* xadj, const int* adj, const double* xyz, int* perm_out,
                       double* stats) {
  if (n <= 0 || !xadj || !adj || !xyz) return TEMF_EARG;
  try {
    std::vector<int64_t> xa(xadj, xadj + n + 1);
    SymbolicOptions o;
    o.max_sn_cols = kSnCols;
    Symbolic S;
    analyse(n, xa.data(), adj, xyz, o, S);
    if (perm_out) std::copy(S.perm.begin(), S.perm.end(), perm_out);
    if (stats) {
      stats[0] = S.n; stats[1] = S.nsn; stats[2] = S.nlevels; stats[3] = (double)S.nnzL;
      stats[4] = (double)S.stored; stats[5] = S.flops; stats[6] = S.t_order;
      stats[7] = S.t_etree + S.t_colcount + S.t_super;
      stats[8] = (double)S.nnzL_exact;
    }
    return TEMF_OK;
  } catch (...) {
    return TEMF_EINTERNAL;
  }
}

int temf_schedule_check(int n, const long long* xadj, const int* adj, const double* xyz, char* msg, int msg_len) {
  if (n <= 0 || !xadj || !adj || !xyz) return TEMF_EARG;
  try {
    std::vector<int64_t> xa(xadj, xadj + n + 1);
    SymbolicOptions o;
    o.max_sn_cols = kSnCols;
    Symbolic S;
    analyse(n, xa.data(), adj, xyz, o, S);
    const std::string w = check_schedules(S);
    if (msg && msg_len > 0) {
      std::strncpy(msg, w.c_str(), msg_len - 1);
      msg[msg_len - 1] = 0;
    }
    return w.empty() ? TEMF_OK : 1;
  } catch (...) {
    return TEMF_EINTERNAL;
  }
}

// ---- PARDISO shim -----------------------------------------------------------
}  // extern "C"

// The structure checks of MKL's sparse matrix checker as pardiso_checker
// (src/FETD_UTILITY.f90:993-1027) configures it: 1-based CSR, ia(1) = 1,
// ia(n+1) - 1 = nnz, ia non-decreasing, column indices in 1..n and strictly
// ascending within a row, and for the symmetric case only the upper
// triangle.  Empty string, or the first violation with its row and position.
static std::string check_user_csr(int symm, int n, int nnz, const int* ia, const int* ja) {
  char buf[160];
  if (n <= 0 || nnz < 0) return "n must be positive and nnz non-negative";
  if (ia[0] != 1) return "ia(1) must be 1 (one-based indexing)";
  if ((long long)ia[n] - 1 != nnz) {
    std::snprintf(buf, sizeof buf, "ia(n+1)-1 = %d differs from nnz = %d", ia[n] - 1, nnz);
    return buf;
  }
  for (int i = 0; i < n; ++i) {
    if (ia[i + 1] < ia[i]) {
      std::snprintf(buf, sizeof buf, "ia decreases at row %d", i + 1);
      return buf;
    }
    for (int q = ia[i] - 1; q < ia[i + 1] - 1; ++q) {
      const int j = ja[q];
      if (j < 1 || j > n) {
        std::snprintf(buf, sizeof buf, "column index %d out of range in row %d (position %d)", j, i + 1, q + 1);
        return buf;
      }
      if (symm && j < i + 1) {
        std::snprintf(buf, sizeof buf, "entry (%d,%d) below the diagonal of an upper-triangular matrix", i + 1, j);
        return buf;
      }
      if (q > ia[i] - 1 && j <= ja[q - 1]) {
        std::snprintf(buf, sizeof buf, "column indices not strictly ascending in row %d (position %d)", i + 1, q + 1);
        return buf;
      }
    }
  }
  return std::string();
}

extern "C" {

int temf_pardiso_checker(int symm, int n, int nnz, const int* ia, const int* ja, int* checker, char* msg,
                         int msg_len) {
  if (!ia || !checker || (nnz > 0 && !ja)) return TEMF_EARG;
  try {
    const std::string w = check_user_csr(symm, n, nnz, ia, ja);
    *checker = w.empty() ? 1 : 0;
    if (msg && msg_len > 0) {
      std::strncpy(msg, w.c_str(), msg_len - 1);
      msg[msg_len - 1] = 0;
    }
    return TEMF_OK;
  } catch (...) {
    return TEMF_EINTERNAL;
  }
}

int temf_pardiso_alloc(temf_ctx* c, int max_matrix) {
  return guarded(c, [&] {
    if (max_matrix < 1 || max_matrix > 2) throw ArgError("maximum number of matrix error (1 or 2 slots)");
    extra(c).shim_max = max_matrix;
    return TEMF_OK;
  });
}

int temf_pardiso_direct_1(temf_ctx* c, int num_m, int symm, int n, int nnz, const int* ia, const int* ja,
                          const double* va) {
  return guarded(c, [&] {
    CtxExtra& X = extra(c);
    if (X.shim_max < 1) throw StateError("call temf_pardiso_alloc first");
    if (num_m < 1 || num_m > X.shim_max) throw ArgError("num_m out of range");
    if (!symm) throw ArgError("only the symmetric (mtype 2) path of the reference is supported");
    need(c->analysed, "temf_pardiso_direct_1: the mesh pattern must be analysed (temf_analyse)");
    if (n != c->n_edges || !ia || !ja || !va || nnz <= 0) throw ArgError("matrix size differs from the mesh");
    {
      const std::string w = check_user_csr(symm, n, nnz, ia, ja);
      if (!w.empty()) throw ArgError("matrix error: " + w);
    }
    if (X.shim_n != n || X.shim_nnz != nnz || X.shim_map.size() != (size_t)nnz) {
      // map each user entry (upper, 1-based) onto the permuted lower pattern
      const Pattern& P = c->pat;
      X.shim_map.assign(nnz, -1);
      X.shim_map_up.assign(nnz, -1);
      for (int i = 0; i < n; ++i) {
        for (int q = ia[i] - 1; q < ia[i + 1] - 1; ++q) {
          const int j = ja[q] - 1;
          int pi = c->sym.iperm[i], pj = c->sym.iperm[j];
          if (pi < pj) std::swap(pi, pj);  // lower triangle of the permuted matrix: row pi, col pj
          const int* b = P.col.data() + P.rowptr[pi];
          const int* e = P.col.data() + P.rowptr[pi + 1];
          const int* f = std::lower_bound(b, e, pj);
          if (f == e || *f != pj) throw ArgError("matrix error: entry outside the mesh's step-matrix pattern");
          X.shim_map[q] = (int)(f - P.col.data());
          if (pi != pj) {  // the same value at (pj, pi): the full symmetric matrix for the refinement
            const int* b2 = P.col.data() + P.rowptr[pj];
            const int* e2 = P.col.data() + P.rowptr[pj + 1];
            const int* f2 = std::lower_bound(b2, e2, pi);
            if (f2 == e2 || *f2 != pi) throw ArgError("matrix error: pattern not symmetric");
            X.shim_map_up[q] = (int)(f2 - P.col.data());
          }
        }
      }
      X.shim_n = n;
      X.shim_nnz = nnz;
      X.shim_map_d.upload(X.shim_map.data(), X.shim_map.size(), c->stream);
      X.shim_map_up_d.upload(X.shim_map_up.data(), X.shim_map_up.size(), c->stream);
    }
    // place the user's values on the permuted full pattern (kept with the
    // slot: the refinement of an indefinite factor applies them)
    DBuf<double> uv;
    uv.upload(va, nnz, c->stream);
    DBuf<double>& full = X.shim_full[num_m - 1];
    if (full.n < (size_t)c->pat.nnz) full.alloc(c->pat.nnz);
    TEMF_CUDA(cudaMemsetAsync(full.p, 0, c->pat.nnz * sizeof(double), c->stream));
    k_scatter_user<<<ceil_div(nnz, 256), 256, 0, c->stream>>>(nnz, X.shim_map_d.p, uv.p, full.p);
    TEMF_CHECK_LAUNCH();
    k_scatter_user<<<ceil_div(nnz, 256), 256, 0, c->stream>>>(nnz, X.shim_map_up_d.p, uv.p, full.p);
    TEMF_CHECK_LAUNCH();
    // not positive definite: the indefinite mode, as the reference retries with
    // mtype -2 (src/FETD_UTILITY.f90:923-935); the positive return is its warning
    return numeric_factor_values_fallback(*c, num_m - 1, full.p, 1.0, nullptr, 0.0);
  });
}

int temf_pardiso_direct_2(temf_ctx* c, int num_m, const double* b, double* x) {
  return guarded(c, [&] {
    CtxExtra& X = extra(c);
    if (num_m < 1 || num_m > std::max(X.shim_max, 1)) throw ArgError("num_m out of range");
    need(c->slots[num_m - 1].valid, "pardiso_direct_2: slot not factored");
    host_solve(c, num_m - 1, 1, b, x, c->n_edges);
    return TEMF_OK;
  });
}

int temf_pardiso_direct_3(temf_ctx* c, int num_m) { return temf_release(c, num_m); }

int temf_pardiso_dealloc(temf_ctx* c) {
  return guarded(c, [&] {
    CtxExtra& X = extra(c);
    X.shim_max = 0;
    c->slots[0].valid = c->slots[1].valid = false;
    return TEMF_OK;
  });
}

}  // extern "C"
