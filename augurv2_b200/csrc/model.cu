// Handle-scoped C ABI: one opaque ab_model per compiled model, the
// counterpart of the generated module the reference's front end loads
// (augur_iface_init / augur_step / augur_cpy / augur_set_pt /
// augur_get_curr_ll, compiler/augur/src/CudaC/CgStInit.hs:474-602, called
// from pyaugur/pyaugur/augurlib.py:445-519), for callers that hold only host
// memory: ab_init_* copies the host inputs into device memory the handle
// owns (as augur_iface_init deep-copies its inputs, cbits/augur_rtmem.c:
// 297-303), ab_step runs whole augur_step sweeps on the caller's stream,
// ab_get_state / ab_set_state move the parameters through host buffers (the
// augur_cpy / augur_set_pt contract), ab_checkpoint / ab_restore save and
// reload the complete sampler state including the iteration counter (so a
// restored chain continues bit for bit), and ab_curr_ll is augur_get_curr_ll.
// Unlike the reference (process-global MCMC state, exit() on error,
// cbits/augur_mcmclib.h:44-45, cbits/augur_util.c:30-36) every handle is
// independent and every call returns a status; the message of a failed call
// is also kept on the handle (ab_model_last_error).
//
// Each sweep is the same sequence of kernel launches the per-family entry
// points make, with the same seeds and iteration numbers, so a handle
// reproduces the results of the Python samplers built on those entry points.
#include <string.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace {

struct Region {
  void* dev;
  size_t bytes;
};

}  // namespace

struct ab_model {
  int kind = 0;
  uint64_t seed = 0;
  uint32_t iteration = 0;
  std::string err;
  std::vector<void*> allocs;

  virtual ~ab_model() {
    for (void* p : allocs) cudaFree(p);
  }
  template <class T>
  int alloc(T** p, size_t n) {
    void* q = nullptr;
    if (n == 0) n = 1;
    AB_CUDA(cudaMalloc(&q, n * sizeof(T)));
    AB_CUDA(cudaMemset(q, 0, n * sizeof(T)));
    allocs.push_back(q);
    *p = static_cast<T*>(q);
    return AB_OK;
  }
  virtual int step(int n, cudaStream_t st) = 0;
  virtual size_t state_bytes() const = 0;
  virtual int get_state(char* host, cudaStream_t st) = 0;
  virtual int set_state(const char* host, cudaStream_t st) = 0;
  virtual std::vector<Region> regions() = 0;          // the device state a checkpoint holds
  virtual int after_restore(cudaStream_t st) = 0;
  virtual int n_ll() const { return 1; }
  virtual int curr_ll(double* host, cudaStream_t st) = 0;
};

namespace ab {
namespace {

int h2d(void* dev, const void* host, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return AB_OK;
  AB_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, st));
  AB_CUDA(cudaStreamSynchronize(st));
  return AB_OK;
}

int d2h(void* host, const void* dev, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return AB_OK;
  AB_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st));
  AB_CUDA(cudaStreamSynchronize(st));
  return AB_OK;
}

// ---- LDA ---------------------------------------------------------------------
struct LdaModel : ab_model {
  int D = 0, K = 0, V = 0, T = 0, Kp = 0;
  int *doc_off = nullptr, *w = nullptr, *z = nullptr, *cnt_dk = nullptr, *cnt_kw = nullptr;
  double *alpha = nullptr, *beta = nullptr, *theta = nullptr, *phiT = nullptr, *ll_out = nullptr;
  unsigned char *scratch = nullptr, *ll_scratch = nullptr;
  ab_lda* runner = nullptr;

  ~LdaModel() override {
    if (runner) ab_lda_destroy(runner);
  }
  int put_phi(const double* phi, cudaStream_t st) {   // phi [K][V] -> phiT [V][Kp]
    std::vector<double> t((size_t)V * Kp, 0.0);
    for (int k = 0; k < K; ++k)
      for (int v = 0; v < V; ++v) t[(size_t)v * Kp + k] = phi[(size_t)k * V + v];
    return h2d(phiT, t.data(), t.size() * sizeof(double), st);
  }
  int step(int n, cudaStream_t st) override {
    int rc = ab_lda_run(runner, n, 1, st);
    if (rc == AB_OK) iteration += (uint32_t)n;
    return rc;
  }
  size_t state_bytes() const override {
    return sizeof(double) * ((size_t)D * K + (size_t)K * V) + sizeof(int) * (size_t)T;
  }
  int get_state(char* host, cudaStream_t st) override {
    int rc = d2h(host, theta, sizeof(double) * (size_t)D * K, st);
    if (rc) return rc;
    std::vector<double> t((size_t)V * Kp);
    rc = d2h(t.data(), phiT, t.size() * sizeof(double), st);
    if (rc) return rc;
    double* phi = reinterpret_cast<double*>(host + sizeof(double) * (size_t)D * K);
    for (int k = 0; k < K; ++k)
      for (int v = 0; v < V; ++v) phi[(size_t)k * V + v] = t[(size_t)v * Kp + k];
    return d2h(host + sizeof(double) * ((size_t)D * K + (size_t)K * V), z, sizeof(int) * (size_t)T, st);
  }
  int set_state(const char* host, cudaStream_t st) override {
    int rc = h2d(theta, host, sizeof(double) * (size_t)D * K, st);
    if (!rc) rc = put_phi(reinterpret_cast<const double*>(host + sizeof(double) * (size_t)D * K), st);
    if (!rc)
      rc = h2d(z, host + sizeof(double) * ((size_t)D * K + (size_t)K * V), sizeof(int) * (size_t)T, st);
    if (!rc) rc = ab_lda_init_state(runner, iteration, st);
    return rc;
  }
  std::vector<Region> regions() override {
    return {{theta, sizeof(double) * (size_t)D * K}, {phiT, sizeof(double) * (size_t)V * Kp},
            {z, sizeof(int) * (size_t)T}};
  }
  int after_restore(cudaStream_t st) override { return ab_lda_init_state(runner, iteration, st); }
  int curr_ll(double* host, cudaStream_t st) override {
    int rc = ab_lda_ll_mod(D, K, V, doc_off, w, z, alpha, beta, theta, phiT, ll_out, ll_scratch, st);
    return rc ? rc : d2h(host, ll_out, sizeof(double), st);
  }
};

// ---- HLR (per-chain engine) --------------------------------------------------
struct HlrModel : ab_model {
  ab_hlr_model m{};
  int C = 0, n_comps = 0, n_idx = 0;
  std::vector<ab_hlr_comp> comps;
  std::vector<int> idx_h, all_h;
  float* X = nullptr;
  int *y = nullptr, *idx_d = nullptr, *all_d = nullptr;
  ab_hlr_comp* comps_d = nullptr;
  double *pars = nullptr, *stats = nullptr, *ll_out = nullptr;
  unsigned char* scratch = nullptr;

  int step(int n, cudaStream_t st) override {
    int rc = ab_hlr_run_chains(&m, comps.data(), comps_d, n_comps, idx_d, idx_h.data(), C, pars, n, iteration,
                               seed, stats, scratch, st);
    if (rc == AB_OK) iteration += (uint32_t)n;
    return rc;
  }
  size_t state_bytes() const override { return sizeof(double) * (size_t)C * (m.D + 2); }
  int get_state(char* host, cudaStream_t st) override { return d2h(host, pars, state_bytes(), st); }
  int set_state(const char* host, cudaStream_t st) override { return h2d(pars, host, state_bytes(), st); }
  std::vector<Region> regions() override {
    return {{pars, state_bytes()}, {stats, sizeof(double) * (size_t)C * n_comps * AB_HLR_STATS}};
  }
  int after_restore(cudaStream_t) override { return AB_OK; }
  int n_ll() const override { return C; }
  int curr_ll(double* host, cudaStream_t st) override {
    // the block of every parameter has every factor of the model in its full
    // conditional: its log density is the joint's
    int rc = ab_hlr_ll_grad(&m, all_d, all_h.data(), (int)all_h.size(), C, pars, ll_out, nullptr, st);
    return rc ? rc : d2h(host, ll_out, sizeof(double) * (size_t)C, st);
  }
};

// ---- Gaussian mixtures -------------------------------------------------------
struct GmmModel : ab_model {
  int N = 0, d = 0, K = 0, Kc = 0, shared = 0, move = 0, df = 0, compat = 1;
  float* Y = nullptr;
  int *z = nullptr, *cnt = nullptr, *shrinks = nullptr, *accepts = nullptr;
  double *mu0 = nullptr, *cov0 = nullptr, *pis = nullptr, *cov = nullptr, *alpha = nullptr, *scale0 = nullptr;
  double *mu = nullptr, *Linv = nullptr, *hdet = nullptr, *sum = nullptr, *obs = nullptr, *prop_cov = nullptr;
  double* ll_out = nullptr;
  unsigned char *stats_scratch = nullptr, *ll_scratch = nullptr, *z_scratch = nullptr;

  int prep_components(cudaStream_t st) {
    return shared ? AB_OK : ab_gmm_prep(K, d, cov, Linv, hdet, st);
  }
  int step(int n, cudaStream_t st) override {
    for (int s = 0; s < n; ++s) {
      const uint32_t it = iteration;
      int rc = AB_OK;
      if (shared) {
        if (move == 0) {
          rc = ab_gmm_stats(N, d, K, Y, z, nullptr, cnt, sum, nullptr, stats_scratch, st);
          if (!rc) rc = ab_gmm_conj_mu(K, d, 1, mu0, cov0, cnt, sum, cov, mu, seed, it, 0, st);
        } else if (move == 1) {
          rc = ab_gmm_eslice(N, d, K, 1, Y, z, mu0, cov0, Linv, hdet, Kc, mu, seed, it, 0, shrinks, st);
        } else {
          rc = ab_gmm_mwg(N, d, K, 1, Y, z, mu0, prop_cov, Linv, hdet, Kc, Kc + 1, compat, mu, seed, it, 0,
                          accepts, st);
        }
      } else {
        rc = ab_gmm_stats(N, d, K, Y, z, nullptr, cnt, sum, nullptr, stats_scratch, st);
        if (!rc) rc = ab_gmm_conj_pis(K, alpha, cnt, pis, seed, it, 0, st);
        if (!rc) rc = ab_gmm_conj_mu(K, d, 0, mu0, cov0, cnt, sum, cov, mu, seed, it, 0, st);
        if (!rc) rc = ab_gmm_stats(N, d, K, Y, z, mu, cnt, nullptr, obs, stats_scratch, st);
        if (!rc) rc = ab_gmm_conj_cov(K, d, df, scale0, cnt, obs, cov, seed, it, 0, st);
        if (!rc) rc = ab_gmm_prep(K, d, cov, Linv, hdet, st);
      }
      if (!rc) rc = ab_gmm_disc_z_screened(N, d, K, shared, Y, pis, mu, Linv, hdet, z, seed, it, 0, z_scratch, st);
      if (rc) return rc;
      iteration += 1;
    }
    return AB_OK;
  }
  // state: pis f64 [K], mu f64 [K][d], cov f64 [K][d][d] (hmvgmm only), z int32 [N]
  size_t state_bytes() const override {
    return sizeof(double) * ((size_t)K + (size_t)K * d + (shared ? 0 : (size_t)K * d * d)) + sizeof(int) * (size_t)N;
  }
  int get_state(char* host, cudaStream_t st) override {
    size_t o = 0;
    int rc = d2h(host + o, pis, sizeof(double) * K, st);
    o += sizeof(double) * K;
    if (!rc) rc = d2h(host + o, mu, sizeof(double) * (size_t)K * d, st);
    o += sizeof(double) * (size_t)K * d;
    if (!shared) {
      if (!rc) rc = d2h(host + o, cov, sizeof(double) * (size_t)K * d * d, st);
      o += sizeof(double) * (size_t)K * d * d;
    }
    if (!rc) rc = d2h(host + o, z, sizeof(int) * (size_t)N, st);
    return rc;
  }
  int set_state(const char* host, cudaStream_t st) override {
    size_t o = 0;
    int rc = h2d(pis, host + o, sizeof(double) * K, st);
    o += sizeof(double) * K;
    if (!rc) rc = h2d(mu, host + o, sizeof(double) * (size_t)K * d, st);
    o += sizeof(double) * (size_t)K * d;
    if (!shared) {
      if (!rc) rc = h2d(cov, host + o, sizeof(double) * (size_t)K * d * d, st);
      o += sizeof(double) * (size_t)K * d * d;
    }
    if (!rc) rc = h2d(z, host + o, sizeof(int) * (size_t)N, st);
    if (!rc) rc = prep_components(st);
    return rc;
  }
  std::vector<Region> regions() override {
    return {{pis, sizeof(double) * K},
            {mu, sizeof(double) * (size_t)K * d},
            {cov, sizeof(double) * (size_t)Kc * d * d},
            {z, sizeof(int) * (size_t)N},
            {shrinks, sizeof(int) * K},
            {accepts, sizeof(int) * K}};
  }
  int after_restore(cudaStream_t st) override { return prep_components(st); }
  int curr_ll(double* host, cudaStream_t st) override {
    int rc = prep_components(st);
    if (!rc)
      rc = ab_gmm_ll_mod(N, d, K, shared, Y, z, pis, mu, Linv, hdet, mu0, Linv + (size_t)Kc * d * d, hdet + Kc,
                         shared ? nullptr : alpha, shared ? 0 : df, shared ? nullptr : scale0,
                         shared ? nullptr : hdet + Kc + 2, ll_out, ll_scratch, st);
    return rc ? rc : d2h(host, ll_out, sizeof(double), st);
  }
};

// Records a failed call's message on the handle as well.
int keep(ab_model* h, int rc) {
  if (rc != AB_OK && h) h->err = ab_last_error();
  return rc;
}

template <class M>
int finish_init(M* h, int rc, ab_model** out) {
  if (rc != AB_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return AB_OK;
}

constexpr uint64_t CKPT_MAGIC = 0x3174706b63626101ull;   // "\x01abckpt1"

struct CkptHeader {
  uint64_t magic;
  int32_t kind, n_regions;
  uint64_t seed;
  uint64_t iteration;
};

}  // namespace
}  // namespace ab

using namespace ab;

extern "C" int ab_init_lda(const ab_lda_init* in, ab_model** out) {
  AB_REQUIRE(in && out, AB_ERR_ARG, "ab_init_lda: null argument");
  AB_REQUIRE(in->D > 0 && in->K > 0 && in->V > 0, AB_ERR_ARG, "ab_init_lda: sizes must be positive");
  AB_REQUIRE(in->doc_off && in->w && in->alpha && in->beta, AB_ERR_ARG, "ab_init_lda: null host array");
  const int D = in->D, K = in->K, V = in->V;
  AB_REQUIRE(in->doc_off[0] == 0, AB_ERR_ARG, "ab_init_lda: doc_off[0] must be 0");
  for (int d = 0; d < D; ++d)
    AB_REQUIRE(in->doc_off[d + 1] >= in->doc_off[d], AB_ERR_ARG, "ab_init_lda: doc_off must be nondecreasing");
  const int T = in->doc_off[D];
  for (int t = 0; t < T; ++t)
    AB_REQUIRE(in->w[t] >= 0 && in->w[t] < V, AB_ERR_ARG, "ab_init_lda: token %d has id %d outside [0, V)", t,
               in->w[t]);
  if (in->z)
    for (int t = 0; t < T; ++t)
      AB_REQUIRE(in->z[t] >= 0 && in->z[t] < K, AB_ERR_ARG, "ab_init_lda: z[%d] outside [0, K)", t);
  LdaModel* h = new LdaModel();
  h->kind = AB_MODEL_LDA;
  h->D = D; h->K = K; h->V = V; h->T = T; h->Kp = ab_lda_phi_stride(K);
  h->seed = in->seed;
  h->iteration = in->iter0;
  cudaStream_t st = nullptr;
  int rc = AB_OK;
  auto chk = [&](int r) { if (rc == AB_OK) rc = r; };
  chk(h->alloc(&h->doc_off, D + 1));
  chk(h->alloc(&h->w, T));
  chk(h->alloc(&h->z, T));
  chk(h->alloc(&h->cnt_dk, (size_t)D * K));
  chk(h->alloc(&h->cnt_kw, (size_t)K * V));
  chk(h->alloc(&h->alpha, K));
  chk(h->alloc(&h->beta, V));
  chk(h->alloc(&h->theta, (size_t)D * K));
  chk(h->alloc(&h->phiT, (size_t)V * h->Kp));
  chk(h->alloc(&h->ll_out, 1));
  chk(h->alloc(&h->scratch, ab_lda_scratch_bytes(K, V)));
  chk(h->alloc(&h->ll_scratch, ab_ll_scratch_bytes()));
  if (rc) return finish_init(h, rc, out);
  chk(h2d(h->doc_off, in->doc_off, sizeof(int) * (D + 1), st));
  chk(h2d(h->w, in->w, sizeof(int) * (size_t)T, st));
  chk(h2d(h->alpha, in->alpha, sizeof(double) * K, st));
  chk(h2d(h->beta, in->beta, sizeof(double) * V, st));
  {
    std::vector<double> th((size_t)D * K, 1.0 / K);
    if (in->theta) memcpy(th.data(), in->theta, th.size() * sizeof(double));
    chk(h2d(h->theta, th.data(), th.size() * sizeof(double), st));
    std::vector<double> ph((size_t)K * V, 1.0 / V);
    if (in->phi) memcpy(ph.data(), in->phi, ph.size() * sizeof(double));
    if (!rc) chk(h->put_phi(ph.data(), st));
  }
  if (in->z) chk(h2d(h->z, in->z, sizeof(int) * (size_t)T, st));
  if (rc) return finish_init(h, rc, out);
  ab_lda_desc desc{};
  desc.D = D; desc.K = K; desc.V = V;
  desc.doc_off = h->doc_off; desc.w = h->w; desc.alpha = h->alpha; desc.beta = h->beta;
  desc.z = h->z; desc.theta = h->theta; desc.phiT = h->phiT; desc.cnt_dk = h->cnt_dk; desc.cnt_kw = h->cnt_kw;
  desc.scratch = h->scratch; desc.seed = in->seed;
  chk(ab_lda_create(&desc, &h->runner));
  if (!rc) chk(ab_lda_init_state(h->runner, h->iteration, st));
  if (!rc) { cudaError_t e = cudaStreamSynchronize(st); if (e != cudaSuccess) rc = cuda_status(e, "ab_init_lda"); }
  return finish_init(h, rc, out);
}

extern "C" int ab_init_hlr(const ab_hlr_init* in, ab_model** out) {
  AB_REQUIRE(in && out, AB_ERR_ARG, "ab_init_hlr: null argument");
  AB_REQUIRE(in->N > 0 && in->D > 0 && in->C > 0 && in->n_comps > 0, AB_ERR_ARG, "ab_init_hlr: bad sizes");
  AB_REQUIRE(in->X && in->y && in->pars && in->comps && in->idx && in->n_idx > 0, AB_ERR_ARG,
             "ab_init_hlr: null host array");
  const int N = in->N, D = in->D, C = in->C;
  for (int i = 0; i < in->n_idx; ++i)
    AB_REQUIRE(in->idx[i] >= 0 && in->idx[i] < D + 2, AB_ERR_ARG, "ab_init_hlr: block index %d outside [0, D+2)",
               in->idx[i]);
  for (int c = 0; c < in->n_comps; ++c)
    AB_REQUIRE(in->comps[c].idx_off >= 0 && in->comps[c].P > 0 && in->comps[c].idx_off + in->comps[c].P <= in->n_idx,
               AB_ERR_ARG, "ab_init_hlr: component %d's block lies outside idx", c);
  HlrModel* h = new HlrModel();
  h->kind = AB_MODEL_HLR;
  h->seed = in->seed;
  h->iteration = in->iter0;
  h->C = C;
  h->n_comps = in->n_comps;
  h->n_idx = in->n_idx;
  h->comps.assign(in->comps, in->comps + in->n_comps);
  h->idx_h.assign(in->idx, in->idx + in->n_idx);
  h->all_h.push_back(D + 1);
  if (in->has_b) h->all_h.push_back(D);
  for (int j = 0; j < D; ++j) h->all_h.push_back(j);
  cudaStream_t st = nullptr;
  int rc = AB_OK;
  auto chk = [&](int r) { if (rc == AB_OK) rc = r; };
  chk(h->alloc(&h->X, (size_t)N * D));
  chk(h->alloc(&h->y, N));
  chk(h->alloc(&h->idx_d, in->n_idx));
  chk(h->alloc(&h->all_d, h->all_h.size()));
  chk(h->alloc(&h->comps_d, in->n_comps));
  chk(h->alloc(&h->pars, (size_t)C * (D + 2)));
  chk(h->alloc(&h->stats, (size_t)C * in->n_comps * AB_HLR_STATS));
  chk(h->alloc(&h->ll_out, C));
  bool nuts = false;
  for (const auto& c : h->comps) nuts = nuts || c.kind == 1;
  chk(h->alloc(&h->scratch, nuts ? ab_hlr_chain_scratch_bytes(C, D) : 8));
  if (rc) return finish_init(h, rc, out);
  {
    std::vector<float> xf((size_t)N * D);
    for (size_t i = 0; i < xf.size(); ++i) xf[i] = (float)in->X[i];
    chk(h2d(h->X, xf.data(), xf.size() * sizeof(float), st));
  }
  chk(h2d(h->y, in->y, sizeof(int) * N, st));
  chk(h2d(h->idx_d, in->idx, sizeof(int) * in->n_idx, st));
  chk(h2d(h->all_d, h->all_h.data(), sizeof(int) * h->all_h.size(), st));
  chk(h2d(h->comps_d, in->comps, sizeof(ab_hlr_comp) * in->n_comps, st));
  chk(h2d(h->pars, in->pars, sizeof(double) * (size_t)C * (D + 2), st));
  ab_hlr_model& m = h->m;
  m.N = N; m.D = D; m.ldx = D; m.has_b = in->has_b; m.vprior = in->vprior; m.compat = in->compat;
  m.x_dtype = AB_F32; m.lam = in->lam; m.a0 = in->a0; m.s0 = in->s0; m.X = h->X; m.y = h->y;
  return finish_init(h, rc, out);
}

extern "C" int ab_init_gmm(const ab_gmm_init* in, ab_model** out) {
  AB_REQUIRE(in && out, AB_ERR_ARG, "ab_init_gmm: null argument");
  AB_REQUIRE(in->N > 0 && in->d > 0 && in->d <= 64 && in->K > 0 && in->K <= 64, AB_ERR_ARG,
             "ab_init_gmm: need N > 0, 0 < d <= 64, 0 < K <= 64");
  AB_REQUIRE(in->Y && in->mu0 && in->cov0 && in->pis && in->covs && in->mu && in->z, AB_ERR_ARG,
             "ab_init_gmm: null host array");
  AB_REQUIRE(in->shared_cov || (in->alpha && in->scale0 && in->df > in->d - 1), AB_ERR_ARG,
             "ab_init_gmm: hmvgmm needs alpha, scale0 and df > d - 1");
  AB_REQUIRE(in->move >= 0 && in->move <= 2 && (in->shared_cov || in->move == 0), AB_ERR_ARG,
             "ab_init_gmm: move must be 0 (conjugate), or 1 (ESlice) / 2 (MWG) for mvgmm");
  AB_REQUIRE(in->move != 2 || in->prop_cov, AB_ERR_ARG, "ab_init_gmm: MWG needs prop_cov");
  const int N = in->N, d = in->d, K = in->K;
  for (int n = 0; n < N; ++n)
    AB_REQUIRE(in->z[n] >= 0 && in->z[n] < K, AB_ERR_ARG, "ab_init_gmm: z[%d] outside [0, K)", n);
  GmmModel* h = new GmmModel();
  h->kind = AB_MODEL_GMM;
  h->seed = in->seed;
  h->iteration = in->iter0;
  h->N = N; h->d = d; h->K = K; h->shared = in->shared_cov ? 1 : 0; h->Kc = h->shared ? 1 : K;
  h->move = in->move; h->df = in->df; h->compat = in->compat;
  const int Kc = h->Kc;
  const size_t dd = (size_t)d * d;
  cudaStream_t st = nullptr;
  int rc = AB_OK;
  auto chk = [&](int r) { if (rc == AB_OK) rc = r; };
  chk(h->alloc(&h->Y, (size_t)N * d));
  chk(h->alloc(&h->z, N));
  chk(h->alloc(&h->cnt, K));
  chk(h->alloc(&h->shrinks, K));
  chk(h->alloc(&h->accepts, K));
  chk(h->alloc(&h->mu0, d));
  chk(h->alloc(&h->cov0, dd));
  chk(h->alloc(&h->pis, K));
  chk(h->alloc(&h->cov, (size_t)Kc * dd));
  chk(h->alloc(&h->alpha, K));
  chk(h->alloc(&h->scale0, dd));
  chk(h->alloc(&h->prop_cov, dd));
  chk(h->alloc(&h->mu, (size_t)K * d));
  chk(h->alloc(&h->Linv, (size_t)(Kc + 3) * dd));
  chk(h->alloc(&h->hdet, Kc + 3));
  chk(h->alloc(&h->sum, (size_t)K * d));
  chk(h->alloc(&h->obs, (size_t)K * dd));
  chk(h->alloc(&h->ll_out, 1));
  chk(h->alloc(&h->stats_scratch, ab_gmm_stats_scratch_bytes(d, K)));
  chk(h->alloc(&h->z_scratch, ab_gmm_z_scratch_bytes(N, d, K)));
  chk(h->alloc(&h->ll_scratch, ab_ll_scratch_bytes()));
  if (rc) return finish_init(h, rc, out);
  {
    std::vector<float> yf((size_t)N * d);
    for (size_t i = 0; i < yf.size(); ++i) yf[i] = (float)in->Y[i];
    chk(h2d(h->Y, yf.data(), yf.size() * sizeof(float), st));
  }
  chk(h2d(h->z, in->z, sizeof(int) * N, st));
  chk(h2d(h->mu0, in->mu0, sizeof(double) * d, st));
  chk(h2d(h->cov0, in->cov0, sizeof(double) * dd, st));
  chk(h2d(h->pis, in->pis, sizeof(double) * K, st));
  chk(h2d(h->cov, in->covs, sizeof(double) * Kc * dd, st));
  chk(h2d(h->mu, in->mu, sizeof(double) * (size_t)K * d, st));
  if (!h->shared) {
    chk(h2d(h->alpha, in->alpha, sizeof(double) * K, st));
    chk(h2d(h->scale0, in->scale0, sizeof(double) * dd, st));
  }
  chk(h2d(h->prop_cov, in->prop_cov ? in->prop_cov : in->cov0, sizeof(double) * dd, st));
  if (rc) return finish_init(h, rc, out);
  // tables: components [0, Kc), mean prior Kc, MWG proposal Kc + 1, scale0 Kc + 2
  chk(ab_gmm_prep(1, d, h->cov0, h->Linv + Kc * dd, h->hdet + Kc, st));
  chk(ab_gmm_prep(1, d, h->prop_cov, h->Linv + (Kc + 1) * dd, h->hdet + Kc + 1, st));
  if (h->shared) chk(ab_gmm_prep(1, d, h->cov, h->Linv, h->hdet, st));
  else chk(ab_gmm_prep(1, d, h->scale0, h->Linv + (Kc + 2) * dd, h->hdet + Kc + 2, st));
  if (!rc) { cudaError_t e = cudaStreamSynchronize(st); if (e != cudaSuccess) rc = cuda_status(e, "ab_init_gmm"); }
  return finish_init(h, rc, out);
}

extern "C" int ab_model_kind(const ab_model* h) { return h ? h->kind : 0; }

extern "C" const char* ab_model_last_error(const ab_model* h) { return h ? h->err.c_str() : ""; }

extern "C" int ab_step(ab_model* h, int n_iters, void* stream) {
  AB_REQUIRE(h, AB_ERR_ARG, "ab_step: null handle");
  if (n_iters < 0) return keep(h, fail(AB_ERR_ARG, "ab_step: n_iters < 0"));
  return keep(h, h->step(n_iters, as_stream(stream)));
}

extern "C" uint32_t ab_iteration(const ab_model* h) { return h ? h->iteration : 0u; }

extern "C" size_t ab_state_bytes(const ab_model* h) { return h ? h->state_bytes() : 0; }

extern "C" int ab_get_state(ab_model* h, void* host, size_t bytes, void* stream) {
  AB_REQUIRE(h, AB_ERR_ARG, "ab_get_state: null handle");
  if (!host || bytes != h->state_bytes())
    return keep(h, fail(AB_ERR_ARG, "ab_get_state: need a host buffer of %zu bytes", h->state_bytes()));
  return keep(h, h->get_state(static_cast<char*>(host), as_stream(stream)));
}

extern "C" int ab_set_state(ab_model* h, const void* host, size_t bytes, void* stream) {
  AB_REQUIRE(h, AB_ERR_ARG, "ab_set_state: null handle");
  if (!host || bytes != h->state_bytes())
    return keep(h, fail(AB_ERR_ARG, "ab_set_state: need a host buffer of %zu bytes", h->state_bytes()));
  return keep(h, h->set_state(static_cast<const char*>(host), as_stream(stream)));
}

extern "C" size_t ab_checkpoint_bytes(ab_model* h) {
  if (!h) return 0;
  size_t n = sizeof(CkptHeader);
  for (const Region& r : h->regions()) n += sizeof(uint64_t) + r.bytes;
  return n;
}

extern "C" int ab_checkpoint(ab_model* h, void* host, size_t bytes, void* stream) {
  AB_REQUIRE(h, AB_ERR_ARG, "ab_checkpoint: null handle");
  if (!host || bytes != ab_checkpoint_bytes(h))
    return keep(h, fail(AB_ERR_ARG, "ab_checkpoint: need a host buffer of %zu bytes", ab_checkpoint_bytes(h)));
  const std::vector<Region> regs = h->regions();
  char* p = static_cast<char*>(host);
  CkptHeader hd{CKPT_MAGIC, h->kind, (int32_t)regs.size(), h->seed, h->iteration};
  memcpy(p, &hd, sizeof(hd));
  p += sizeof(hd);
  for (const Region& r : regs) {
    const uint64_t n = r.bytes;
    memcpy(p, &n, sizeof(n));
    p += sizeof(n);
    int rc = d2h(p, r.dev, r.bytes, as_stream(stream));
    if (rc) return keep(h, rc);
    p += r.bytes;
  }
  return AB_OK;
}

extern "C" int ab_restore(ab_model* h, const void* host, size_t bytes, void* stream) {
  AB_REQUIRE(h, AB_ERR_ARG, "ab_restore: null handle");
  if (!host || bytes != ab_checkpoint_bytes(h))
    return keep(h, fail(AB_ERR_ARG, "ab_restore: the checkpoint has %zu bytes, this model's have %zu", bytes,
                        ab_checkpoint_bytes(h)));
  const char* p = static_cast<const char*>(host);
  CkptHeader hd;
  memcpy(&hd, p, sizeof(hd));
  p += sizeof(hd);
  const std::vector<Region> regs = h->regions();
  if (hd.magic != CKPT_MAGIC || hd.kind != h->kind || hd.n_regions != (int32_t)regs.size())
    return keep(h, fail(AB_ERR_ARG, "ab_restore: not a checkpoint of this kind of model"));
  for (const Region& r : regs) {
    uint64_t n;
    memcpy(&n, p, sizeof(n));
    p += sizeof(n);
    if (n != r.bytes) return keep(h, fail(AB_ERR_ARG, "ab_restore: checkpoint sizes differ from this model's"));
    int rc = h2d(r.dev, p, r.bytes, as_stream(stream));
    if (rc) return keep(h, rc);
    p += r.bytes;
  }
  if (h->kind == AB_MODEL_LDA && hd.seed != h->seed)   // the sweep graph bakes the seed in
    return keep(h, fail(AB_ERR_ARG, "ab_restore: an LDA checkpoint restores into a model with its seed"));
  h->seed = hd.seed;
  h->iteration = (uint32_t)hd.iteration;
  return keep(h, h->after_restore(as_stream(stream)));
}

extern "C" int ab_curr_ll_count(const ab_model* h) { return h ? h->n_ll() : 0; }

extern "C" int ab_curr_ll(ab_model* h, double* host, int n, void* stream) {
  AB_REQUIRE(h, AB_ERR_ARG, "ab_curr_ll: null handle");
  if (!host || n != h->n_ll())
    return keep(h, fail(AB_ERR_ARG, "ab_curr_ll: need room for %d values", h->n_ll()));
  return keep(h, h->curr_ll(host, as_stream(stream)));
}

extern "C" int ab_destroy(ab_model* h) {
  delete h;
  return AB_OK;
}
