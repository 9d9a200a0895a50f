// Batched execution (tti_batch_*): many shots, of one model or of several
// models of different sizes, advanced together. Every half-step is one launch
// over all instances' tiles, driven by a CTA -> (instance, tile) work table;
// instances of one model share its parameter arrays, and the table lists the
// instances of a model tile by tile so that the shots reading one parameter
// tile run together and reuse it from L2. The time index lives in a device
// step counter, so the launches of G steps are captured once in a CUDA graph
// and the graph is replayed for the whole loop.
#include <algorithm>
#include <chrono>
#include <thread>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tiled.cuh"

using namespace ttifd;

struct tti_batch {
  int device = 0;
  int variant = 0;
  bool exact = false;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<tti_handle *> models;  // model m's handle is also its first instance
  std::vector<tti_handle *> inst;
  std::vector<int> model_of;
  int max_nt = 0, max_Nx = 0;
  bool any_vsrc = false;
  bool square = false;  // every instance uses the folded coefficients (FMA mode, dx == dz)
  // device tables (fixed addresses: a captured graph refers to them)
  tiled::HalfArgs *d_vel = nullptr, *d_str = nullptr;
  tiled::Work *d_work = nullptr;
  int nwork = 0;
  BatchPost *d_post = nullptr;
  BatchSrc *d_src = nullptr;
  SourceTables *d_tab = nullptr;
  int *d_step = nullptr;
  int group = 0;  // work-table order: shots of a model interleaved tile by tile in groups of `group` (0: all)
  bool persistent = false;  // one resident wave of CTAs walks the work table (else one CTA per item)
  int graph_steps = 20;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int steps_done = 0;
  float last_ms = 0.0f;
  long long launches = 0;
  std::string err;
};

namespace {

thread_local std::string g_batch_create_error;

int berr(tti_batch *b, int code, const char *fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  else g_batch_create_error = buf;
  return code;
}

#define BCK(b, call)                                                                                   \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) {                                                                           \
      cudaGetLastError();                                                                              \
      return berr((b), e_ == cudaErrorMemoryAllocation ? TTI_ERR_NOMEM : TTI_ERR_CUDA, "%s: %s", #call, \
                  cudaGetErrorString(e_));                                                             \
    }                                                                                                  \
  } while (0)

// Instances read their model's state: uploaded or not, the undamped-tile flag,
// and (for the gradient's chain rule) the model's epsilon, delta, theta.
void sync_instances(tti_batch *b)
{
  for (size_t i = 0; i < b->inst.size(); ++i) {
    tti_handle *h = b->inst[i];
    const tti_handle *mh = b->models[b->model_of[i]];
    h->have_model = mh->have_model;
    h->undamped_ok = mh->undamped_ok;
    if (h != mh) {
      h->m_eps = mh->m_eps;
      h->m_delta = mh->m_delta;
      h->m_theta = mh->m_theta;
    }
  }
}

// dst[i] += src[i], i < n
__global__ void k_accumulate(float *dst, const float *src, size_t n)
{
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] += src[i];
}

// Fills the device tables from the instances' current sources and receivers.
int build_tables(tti_batch *b)
{
  const int n = (int)b->inst.size(), nm = (int)b->models.size();
  std::vector<tiled::HalfArgs> vel(n), str(n);
  std::vector<BatchPost> post(n);
  std::vector<BatchSrc> src(n);
  std::vector<SourceTables> tab(nm);
  for (int m = 0; m < nm; ++m) handle_source_tables(b->models[m], &tab[m]);
  std::vector<int> tiles(n);
  bool all_square = true;
  sync_instances(b);
  for (int i = 0; i < n; ++i) {
    tti_handle *h = b->inst[i];
    const tti_config &c = h->cfg;
    const StepArgs a = handle_step_args(h);
    const CUtensorMap *tm = static_cast<const CUtensorMap *>(h->tmaps);
    tiled::HalfArgs ha{};
    memset(&ha, 0, sizeof ha);
    ha.g = h->g;
    ha.f = a.f;
    ha.p = a.p;
    ha.pk = packed::Packed{h->pk_cf, h->pk_vsc, h->pk_sc, h->pk_c4};
    ha.invdx = h->invdx;
    ha.invdz = h->invdz;
    ha.dt = c.dt;
    const dim3 gr = tiled::grid(h->g, &ha.z_base);
    ha.x_base = NH;
    ha.undamped_ok = h->undamped_ok;
    ha.freesurface = c.freesurface;
    tiled::set_square(ha, b->exact);
    all_square = all_square && ha.square;
    ha.wait_limit = h->wait_limit;
    ha.err = h->d_flag;
    ha.nt = c.nt;
    ha.tiles_z = (int)gr.x;
    tiles[i] = (int)(gr.x * gr.y);
    vel[i] = ha;
    vel[i].map[0] = tm[2];
    vel[i].map[1] = tm[3];
    vel[i].map[2] = tm[4];
    str[i] = ha;
    str[i].map[0] = tm[0];
    str[i].map[1] = tm[1];
    SourceSet s{h->nsrc, h->d_sx, h->d_sz, h->d_src, c.nt};
    BatchPost &bp = post[i];
    memset(&bp, 0, sizeof bp);
    bp.g = h->g;
    bp.f = a.f;
    bp.p.freesurface = c.freesurface;
    bp.p.stype = s.n > 0 && c.stype == 1 ? 1 : 0;
    bp.p.tensor = c.variant == TTI_TENSOR;
    bp.p.src = s;
    memcpy(bp.p.k1, tab[b->model_of[i]].k1, sizeof bp.p.k1);
    const bool want_v = c.seistype == 1 || c.seistype == 3, want_p = c.seistype == 2 || c.seistype == 3;
    for (int k = 0; k < 3; ++k) {
      const bool on = (k < 2 ? want_v : want_p) && h->nrec[k] > 0;
      bp.p.colptr[k] = on ? h->d_rcol[k] : nullptr;
      bp.p.rz[k] = h->d_rzs[k];
      bp.p.rid[k] = h->d_rid[k];
      bp.p.rec[k] = h->d_rec[k];
      bp.p.nrec[k] = h->nrec[k];
    }
    bp.p.flag = h->d_flag;
    bp.nt = c.nt;
    bp.mode2 = c.mode == 2;
    bp.mt = c.mt;
    bp.rec_on = c.seistype > 0 && h->nrec[0] + h->nrec[1] + h->nrec[2] > 0;
    BatchSrc &bs = src[i];
    memset(&bs, 0, sizeof bs);
    bs.g = h->g;
    bs.f = a.f;
    bs.s = s;
    bs.tab = b->d_tab + b->model_of[i];
    bs.variant = c.variant;
    bs.stype = c.stype >= 2 ? c.stype : 0;
    bs.nt = c.nt;
    bs.mode2 = c.mode == 2;
  }
  // work table: per model, per group of its instances, tile by tile
  std::vector<tiled::Work> work;
  work.reserve(b->nwork);
  for (int m = 0; m < nm; ++m) {
    std::vector<int> mine;
    for (int i = 0; i < n; ++i)
      if (b->model_of[i] == m) mine.push_back(i);
    const int G = b->group > 0 ? b->group : (int)mine.size();
    for (size_t g0 = 0; g0 < mine.size(); g0 += G)
      for (int t = 0; t < tiles[mine[0]]; ++t)
        for (size_t k = g0; k < std::min(mine.size(), g0 + G); ++k) work.push_back(tiled::Work{mine[k], t});
  }
  if ((int)work.size() != b->nwork) return berr(b, TTI_ERR_STATE, "work table size changed");
  if (all_square != b->square && b->exec) {  // the captured launches select the kernels
    cudaGraphExecDestroy(b->exec);
    cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
  }
  b->square = all_square;
  BCK(b, cudaMemcpyAsync(b->d_vel, vel.data(), sizeof(tiled::HalfArgs) * n, cudaMemcpyHostToDevice, b->stream));
  BCK(b, cudaMemcpyAsync(b->d_str, str.data(), sizeof(tiled::HalfArgs) * n, cudaMemcpyHostToDevice, b->stream));
  BCK(b, cudaMemcpyAsync(b->d_post, post.data(), sizeof(BatchPost) * n, cudaMemcpyHostToDevice, b->stream));
  BCK(b, cudaMemcpyAsync(b->d_src, src.data(), sizeof(BatchSrc) * n, cudaMemcpyHostToDevice, b->stream));
  BCK(b, cudaMemcpyAsync(b->d_tab, tab.data(), sizeof(SourceTables) * nm, cudaMemcpyHostToDevice, b->stream));
  BCK(b, cudaMemcpyAsync(b->d_work, work.data(), sizeof(tiled::Work) * work.size(), cudaMemcpyHostToDevice,
                         b->stream));
  BCK(b, cudaStreamSynchronize(b->stream));
  return TTI_OK;
}

// Launch description of a half-step (`vel`: the velocity tables, else the stress ones).
tiled::BatchLaunch batch_launch(const tti_batch *b, bool vel)
{
  return tiled::BatchLaunch{vel ? b->d_vel : b->d_str, b->d_work, b->nwork, b->d_step, b->variant, b->exact,
                            b->square, b->persistent};
}

// The launches of one time step (all instances).
int launch_step(tti_batch *b)
{
  const int n = (int)b->inst.size();
  BCK(b, tiled::launch_velocity_batch(batch_launch(b, true), b->stream));
  if (b->any_vsrc) launch_sources_batch(b->d_src, n, b->d_step, b->stream);
  BCK(b, tiled::launch_stress_batch(batch_launch(b, false), b->stream));
  launch_post_batch(b->d_post, n, b->max_Nx, b->d_step, b->stream);
  launch_advance(b->d_step, b->stream);
  BCK(b, cudaGetLastError());
  return TTI_OK;
}

int launches_per_step(const tti_batch *b) { return 4 + (b->any_vsrc ? 1 : 0); }

int ensure_graph(tti_batch *b)
{
  if (b->exec || b->graph_steps <= 0) return TTI_OK;
  BCK(b, tiled::prepare_batch(batch_launch(b, true)));
  BCK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = TTI_OK;
  for (int k = 0; k < b->graph_steps && rc == TTI_OK; ++k) rc = launch_step(b);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return berr(b, TTI_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  b->graph = g;
  BCK(b, cudaGraphInstantiate(&b->exec, g, 0));
  return TTI_OK;
}

int check_flags(tti_batch *b)
{
  for (size_t i = 0; i < b->inst.size(); ++i) {
    const int rc = handle_check_flag(b->inst[i]);
    if (rc) return berr(b, rc, "instance %zu: %s", i, b->inst[i]->err.c_str());
  }
  return TTI_OK;
}

}  // namespace

extern "C" {

const char *tti_batch_last_error(const tti_batch *b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

int tti_batch_destroy(tti_batch *b)
{
  if (!b) return TTI_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (size_t i = 0; i < b->inst.size(); ++i)  // shared instances before their models
    if (b->inst[i] && b->inst[i]->owner) tti_destroy(b->inst[i]);
  for (auto h : b->models) tti_destroy(h);
  cudaFree(b->d_vel);
  cudaFree(b->d_str);
  cudaFree(b->d_work);
  cudaFree(b->d_post);
  cudaFree(b->d_src);
  cudaFree(b->d_tab);
  cudaFree(b->d_step);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return TTI_OK;
}

int tti_batch_create(tti_batch **out, int nmodels, const tti_config *cfg, int ninst, const int *model_of, int device)
{
  if (!out || !cfg || nmodels < 1 || ninst < 1)
    return berr(nullptr, TTI_ERR_ARG, "tti_batch_create: need at least one model and one instance");
  *out = nullptr;
  for (int m = 0; m < nmodels; ++m) {
    if (cfg[m].variant != cfg[0].variant)
      return berr(nullptr, TTI_ERR_ARG, "all models of a batch use the same formulation");
    if (cfg[m].wsave != 0 || cfg[m].energy != 0)
      return berr(nullptr, TTI_ERR_ARG, "batched runs record traces only (wsave = 0, energy = 0)");
  }
  std::vector<int> first(nmodels, -1);
  for (int i = 0; i < ninst; ++i) {
    const int m = model_of ? model_of[i] : 0;
    if (m < 0 || m >= nmodels) return berr(nullptr, TTI_ERR_ARG, "instance %d: model %d out of range", i, m);
    if (first[m] < 0) first[m] = i;
  }
  for (int m = 0; m < nmodels; ++m)
    if (first[m] < 0) return berr(nullptr, TTI_ERR_ARG, "model %d has no instance", m);
  tti_batch *b = new tti_batch();
  b->device = device;
  b->variant = cfg[0].variant;
  const char *ex = getenv("TTIFD_EXACT");  // the handles' default: the reference's rounding
  b->exact = !(ex && ex[0] == '0');
  const char *gs = getenv("TTIFD_GRAPH_STEPS");
  if (gs) b->graph_steps = atoi(gs);
  auto fail = [&](int rc, const std::string &msg) {
    tti_batch_destroy(b);
    return berr(nullptr, rc, "%s", msg.c_str());
  };
  int rc = TTI_OK;
  b->models.assign(nmodels, nullptr);
  b->inst.assign(ninst, nullptr);
  b->model_of.resize(ninst);
  for (int m = 0; m < nmodels; ++m) {
    if ((rc = create_handle(&b->models[m], &cfg[m], device, nullptr, true)))
      return fail(rc, tti_last_error(nullptr));
    b->inst[first[m]] = b->models[m];
  }
  for (int i = 0; i < ninst; ++i) {
    const int m = model_of ? model_of[i] : 0;
    b->model_of[i] = m;
    if (!b->inst[i] && (rc = create_handle(&b->inst[i], &cfg[m], device, b->models[m], true)))
      return fail(rc, tti_last_error(nullptr));
  }
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess)
    return fail(TTI_ERR_CUDA, "stream/event creation failed");
  b->nwork = 0;
  for (int i = 0; i < ninst; ++i) {
    int zb;
    const dim3 gr = tiled::grid(b->inst[i]->g, &zb);
    b->nwork += (int)(gr.x * gr.y);
    b->max_nt = std::max(b->max_nt, b->inst[i]->cfg.nt);
    b->max_Nx = std::max(b->max_Nx, b->inst[i]->g.Nx);
    b->any_vsrc = b->any_vsrc || b->inst[i]->cfg.stype >= 2;
  }
  const bool ok = cudaMalloc(&b->d_vel, sizeof(tiled::HalfArgs) * ninst) == cudaSuccess &&
                  cudaMalloc(&b->d_str, sizeof(tiled::HalfArgs) * ninst) == cudaSuccess &&
                  cudaMalloc(&b->d_post, sizeof(BatchPost) * ninst) == cudaSuccess &&
                  cudaMalloc(&b->d_src, sizeof(BatchSrc) * ninst) == cudaSuccess &&
                  cudaMalloc(&b->d_tab, sizeof(SourceTables) * nmodels) == cudaSuccess &&
                  cudaMalloc(&b->d_work, sizeof(tiled::Work) * (size_t)std::max(1, b->nwork)) == cudaSuccess &&
                  cudaMalloc(&b->d_step, sizeof(int)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    return fail(TTI_ERR_NOMEM, "device allocation of the batch tables failed");
  }
  *out = b;
  return TTI_OK;
}

tti_handle *tti_batch_instance(tti_batch *b, int i)
{
  if (!b || i < 0 || i >= (int)b->inst.size()) return nullptr;
  return b->inst[i];
}

int tti_batch_upload_model(tti_batch *b, int m, const float *vp, const float *vs, const float *rho,
                           const float *epsilon, const float *delta, const float *theta)
{
  if (!b || m < 0 || m >= (int)b->models.size()) return berr(b, TTI_ERR_ARG, "model index out of range");
  const int rc = tti_upload_model(b->models[m], vp, vs, rho, epsilon, delta, theta);
  if (rc) return berr(b, rc, "model %d: %s", m, tti_last_error(b->models[m]));
  sync_instances(b);  // the model's instances may now take observed traces
  return TTI_OK;
}

int tti_batch_set_order(tti_batch *b, int group, int graph_steps)
{
  if (!b || group < 0 || graph_steps < 0) return berr(b, TTI_ERR_ARG, "bad batch schedule");
  b->group = group;
  if (graph_steps != b->graph_steps) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_steps = graph_steps;
  }
  return TTI_OK;
}

int tti_batch_set_schedule(tti_batch *b, int persistent)
{
  if (!b || persistent < 0 || persistent > 1) return berr(b, TTI_ERR_ARG, "grid schedule must be 0 or 1");
  if ((persistent == 1) != b->persistent) {  // the captured launches set the grid sizes
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->persistent = persistent == 1;
  }
  return TTI_OK;
}

int tti_batch_get_schedule(const tti_batch *b, int *group, int *graph_steps, int *persistent)
{
  if (!b) return TTI_ERR_ARG;
  if (group) *group = b->group;
  if (graph_steps) *graph_steps = b->graph_steps;
  if (persistent) *persistent = b->persistent ? 1 : 0;
  return TTI_OK;
}

int tti_batch_reset(tti_batch *b)
{
  if (!b) return TTI_ERR_ARG;
  BCK(b, cudaSetDevice(b->device));
  for (size_t m = 0; m < b->models.size(); ++m)
    if (!b->models[m]->have_model) return berr(b, TTI_ERR_STATE, "model %zu not uploaded", m);
  for (auto h : b->inst) {
    const int rc = tti_reset(h);
    if (rc) return berr(b, rc, "%s", tti_last_error(h));
    BCK(b, cudaStreamSynchronize(h->stream));
  }
  int rc = build_tables(b);
  if (rc) return rc;
  BCK(b, cudaMemsetAsync(b->d_step, 0, sizeof(int), b->stream));
  BCK(b, cudaStreamSynchronize(b->stream));
  b->steps_done = 0;
  return TTI_OK;
}

int tti_batch_step(tti_batch *b, int nsteps)
{
  if (!b || nsteps < 0) return TTI_ERR_ARG;
  if (b->steps_done + nsteps > b->max_nt) return berr(b, TTI_ERR_STATE, "step past the longest instance's nt");
  BCK(b, cudaSetDevice(b->device));
  int rc = ensure_graph(b);
  if (rc) return rc;
  BCK(b, cudaEventRecord(b->ev0, b->stream));
  int left = nsteps;
  while (b->exec && left >= b->graph_steps) {
    BCK(b, cudaGraphLaunch(b->exec, b->stream));
    b->launches += (long long)b->graph_steps * launches_per_step(b);
    left -= b->graph_steps;
  }
  for (; left > 0; --left) {
    if ((rc = launch_step(b))) return rc;
    b->launches += launches_per_step(b);
  }
  BCK(b, cudaEventRecord(b->ev1, b->stream));
  BCK(b, cudaEventSynchronize(b->ev1));
  BCK(b, cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
  b->steps_done += nsteps;
  for (auto h : b->inst) h->step_index = std::min(b->steps_done, h->cfg.nt);
  return check_flags(b);
}

int tti_batch_run(tti_batch *b)
{
  int rc = tti_batch_reset(b);
  if (rc) return rc;
  return tti_batch_step(b, b->max_nt);
}

int tti_batch_autotune(tti_batch *b, int nsteps, int *group, int *graph_steps, float *ms_per_step)
{
  if (!b || nsteps < 1) return berr(b, TTI_ERR_ARG, "autotune needs at least one step");
  nsteps = std::min(nsteps, b->max_nt);
  int ninst_max = 0;  // largest number of instances of one model
  for (size_t m = 0; m < b->models.size(); ++m)
    ninst_max = std::max(ninst_max, (int)std::count(b->model_of.begin(), b->model_of.end(), (int)m));
  std::vector<int> groups = {0};
  for (int g : {1, 4, 16})
    if (g < ninst_max) groups.push_back(g);
  const int graphs[] = {0, 20};
  const int NS = 2;  // grids: one CTA per tile, or a persistent wave
  // Each candidate is timed twice, in two rounds over all of them, and keeps
  // its faster time; a graph candidate is timed over at least one replay of
  // its graph (the step loop only replays it when that many steps remain).
  const int warm = std::min(2, nsteps);
  std::vector<float> t_best(groups.size() * 2 * NS, -1.0f);
  for (int round = 0; round < 2; ++round)
    for (int ts = 0; ts < NS; ++ts)
      for (size_t gi = 0; gi < groups.size(); ++gi)
        for (int q = 0; q < 2; ++q) {
          const int g = groups[gi], gs = graphs[q];
          int timed = nsteps - warm;
          if (gs > 0) timed = std::max(timed, gs);
          timed = std::min(timed, b->max_nt - warm);
          if (timed <= 0) continue;
          int rc = tti_batch_set_order(b, g, gs);
          if (!rc) rc = tti_batch_set_schedule(b, ts);
          if (!rc) rc = tti_batch_reset(b);
          if (!rc) rc = tti_batch_step(b, warm);  // warm-up (and graph instantiation)
          if (!rc) rc = tti_batch_step(b, timed);
          if (rc) return rc;
          const float t = b->last_ms / timed;
          float &tb = t_best[(ts * groups.size() + gi) * 2 + q];
          if (tb < 0 || t < tb) tb = t;
        }
  float best = -1.0f;
  int bg = 0, bs = 20, bt = 0;
  for (int ts = 0; ts < NS; ++ts)
    for (size_t gi = 0; gi < groups.size(); ++gi)
      for (int q = 0; q < 2; ++q) {
        const float t = t_best[(ts * groups.size() + gi) * 2 + q];
        if (t >= 0 && (best < 0 || t < best)) {
          best = t;
          bg = groups[gi];
          bs = graphs[q];
          bt = ts;
        }
      }
  int rc = tti_batch_set_order(b, bg, bs);
  if (!rc) rc = tti_batch_set_schedule(b, bt);
  if (!rc) rc = tti_batch_reset(b);
  if (rc) return rc;
  if (group) *group = bg;
  if (graph_steps) *graph_steps = bs;
  if (ms_per_step) *ms_per_step = best;
  return TTI_OK;
}

int tti_batch_grad_run(tti_batch *b, int snapshots, int keep_steps, double *misfits)
{
  if (!b || snapshots < 0 || keep_steps < 1) return berr(b, TTI_ERR_ARG, "bad gradient schedule");
  BCK(b, cudaSetDevice(b->device));
  for (size_t m = 0; m < b->models.size(); ++m)
    if (!b->models[m]->have_model) return berr(b, TTI_ERR_STATE, "model %zu not uploaded", m);
  sync_instances(b);
  const int n = (int)b->inst.size();
  std::vector<int> rc(n, TTI_OK);
  std::vector<double> J(n, 0.0);
  const auto t0 = std::chrono::steady_clock::now();
  {
    // one host thread per instance: each drives its own stream, so the
    // kernels of different shots overlap on the device
    std::vector<std::thread> th;
    th.reserve(n);
    for (int i = 0; i < n; ++i)
      th.emplace_back([&, i] {
        cudaSetDevice(b->device);
        rc[i] = tti_grad_run_binomial(b->inst[i], snapshots, keep_steps, &J[i]);
      });
    for (auto &t : th) t.join();
  }
  for (int i = 0; i < n; ++i)
    if (rc[i]) return berr(b, rc[i], "instance %d: %s", i, tti_last_error(b->inst[i]));
  // the instances' sums into their model's first instance, the others cleared
  for (size_t m = 0; m < b->models.size(); ++m) {
    tti_handle *mh = b->models[m];
    float *dst[7];
    size_t cnt = 0;
    if (tti_grad_accumulators(mh, dst, &cnt, nullptr)) return berr(b, TTI_ERR_STATE, "%s", tti_last_error(mh));
    for (int i = 0; i < n; ++i) {
      tti_handle *h = b->inst[i];
      if (b->model_of[i] != (int)m || h == mh) continue;
      float *src[7];
      if (tti_grad_accumulators(h, src, nullptr, nullptr)) return berr(b, TTI_ERR_STATE, "%s", tti_last_error(h));
      for (int k = 0; k < 7; ++k) {
        k_accumulate<<<1184, 256, 0, mh->stream>>>(dst[k], src[k], cnt);
        BCK(b, cudaMemsetAsync(src[k], 0, cnt * sizeof(float), mh->stream));
      }
      b->launches += 7;
    }
    BCK(b, cudaGetLastError());
    BCK(b, cudaStreamSynchronize(mh->stream));
  }
  b->last_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (misfits)
    for (int i = 0; i < n; ++i) misfits[i] = J[i];
  return TTI_OK;
}

int tti_batch_elapsed_ms(const tti_batch *b, float *ms)
{
  if (!b || !ms) return TTI_ERR_ARG;
  *ms = b->last_ms;
  return TTI_OK;
}

int tti_batch_kernel_launches(const tti_batch *b, long long *n)
{
  if (!b || !n) return TTI_ERR_ARG;
  *n = b->launches;
  return TTI_OK;
}

}  // extern "C"
