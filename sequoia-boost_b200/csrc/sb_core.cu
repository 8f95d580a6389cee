// sb_core.cu — errors, contexts, parameters and model handles.
#include <cstdarg>
#include <cstring>

#include <map>
#include <mutex>

#include "sb_internal.cuh"

namespace sb {

static thread_local std::string g_last_error = "ok";

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int cuda_status(cudaError_t e, const char* what, const char* file, int line) {
  set_error("%s:%d: %s failed: %s", file, line, what, cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return SB_ERR_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
    return SB_ERR_NO_DEVICE;
  return SB_ERR_CUDA;
}

int dalloc(sb_ctx* ctx, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return SB_OK;
  cudaError_t e = cudaMallocAsync(p, bytes, ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return SB_ERR_OOM;
  }
  return SB_OK;
}

int raise_smem_limit(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> set;
  int dev = 0;
  SB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = set[std::make_pair(func, dev)];
  if (bytes <= cur) return SB_OK;
  SB_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  cur = bytes;
  return SB_OK;
}

void dfree(sb_ctx* ctx, void* p) {
  if (p) cudaFreeAsync(p, ctx->stream);
}

int n_outputs(int objective, int num_class) {
  return (objective == SB_OBJ_SOFTMAX || objective == SB_OBJ_SOFTPROB) ? num_class : 1;
}

}  // namespace sb

extern "C" {

const char* sb_last_error(void) { return sb::g_last_error.c_str(); }
const char* sb_version(void) { return "sequoia-boost-b200 0.1.0 (sm_100a)"; }

void sb_train_params_default(sb_train_params* p) {  // config/params.rs:153-186
  std::memset(p, 0, sizeof(*p));
  p->seed = 0;
  p->eta = 0.3;
  p->gamma = 0.0;
  p->min_child_weight = 1.0;
  p->max_delta_step = 0.0;
  p->subsample = 1.0;
  p->colsample_bytree = 1.0;
  p->colsample_bylevel = 1.0;
  p->colsample_bynode = 1.0;
  p->lambda = 1.0;
  p->alpha = 0.0;
  p->scale_pos_weight = 1.0;
  p->objective = SB_OBJ_SQUARED_ERROR;
  p->num_class = 0;
  p->has_base_score = 0;
  p->max_depth = 6;
  p->max_leaves = 0;
  p->grow_policy = SB_GROW_DEPTHWISE;
  p->max_bin = 256;
  p->hist_precision = SB_HIST_FIXED;  // exact, run-to-run deterministic histograms
  p->quantize_bits = 0;
}

int sb_train_params_validate(const sb_train_params* p) {  // config/params.rs:197-261
  SB_REQUIRE(p != nullptr, SB_ERR_INVALID_ARG, "params is NULL");
  auto unit = [](double v) { return v >= 0.0 && v <= 1.0; };
  auto pos = [](double v) { return !std::isnan(v) && v > 0.0; };
  auto nonneg = [](double v) { return !std::isnan(v) && v >= 0.0; };
  SB_REQUIRE(pos(p->eta), SB_ERR_INVALID_ARG, "invalid parameter `eta`: must be > 0, got %g", p->eta);
  SB_REQUIRE(nonneg(p->gamma), SB_ERR_INVALID_ARG, "invalid parameter `gamma`: must be >= 0");
  SB_REQUIRE(nonneg(p->min_child_weight), SB_ERR_INVALID_ARG,
             "invalid parameter `min_child_weight`: must be >= 0");
  SB_REQUIRE(nonneg(p->max_delta_step), SB_ERR_INVALID_ARG,
             "invalid parameter `max_delta_step`: must be >= 0");
  SB_REQUIRE(nonneg(p->lambda), SB_ERR_INVALID_ARG, "invalid parameter `lambda`: must be >= 0");
  SB_REQUIRE(nonneg(p->alpha), SB_ERR_INVALID_ARG, "invalid parameter `alpha`: must be >= 0");
  SB_REQUIRE(pos(p->scale_pos_weight), SB_ERR_INVALID_ARG,
             "invalid parameter `scale_pos_weight`: must be > 0");
  SB_REQUIRE(unit(p->subsample) && p->subsample > 0.0, SB_ERR_INVALID_ARG,
             "invalid parameter `subsample`: must be in (0, 1]");
  SB_REQUIRE(unit(p->colsample_bytree), SB_ERR_INVALID_ARG,
             "invalid parameter `colsample_bytree`: must be in [0, 1]");
  SB_REQUIRE(unit(p->colsample_bylevel), SB_ERR_INVALID_ARG,
             "invalid parameter `colsample_bylevel`: must be in [0, 1]");
  SB_REQUIRE(unit(p->colsample_bynode), SB_ERR_INVALID_ARG,
             "invalid parameter `colsample_bynode`: must be in [0, 1]");
  SB_REQUIRE(p->max_bin >= 2, SB_ERR_INVALID_ARG, "invalid parameter `max_bin`: must be >= 2");
  SB_REQUIRE(!(p->grow_policy == SB_GROW_LOSSGUIDE && p->max_leaves == 0 && p->max_depth == 0),
             SB_ERR_INVALID_ARG,
             "invalid parameter `max_leaves`: lossguide growth needs a bound: set max_leaves or max_depth > 0");
  SB_REQUIRE(p->objective >= SB_OBJ_SQUARED_ERROR && p->objective <= SB_OBJ_SOFTPROB,
             SB_ERR_INVALID_ARG, "unknown objective %d", p->objective);
  SB_REQUIRE(!((p->objective == SB_OBJ_SOFTMAX || p->objective == SB_OBJ_SOFTPROB) && p->num_class < 2),
             SB_ERR_INVALID_ARG, "invalid parameter `num_class`: multiclass objectives require num_class >= 2");
  SB_REQUIRE(p->max_depth >= 0 && p->max_leaves >= 0, SB_ERR_INVALID_ARG, "negative tree limit");
  SB_REQUIRE(p->hist_precision == SB_HIST_FP32 || p->hist_precision == SB_HIST_FIXED,
             SB_ERR_INVALID_ARG, "unknown hist_precision %d", p->hist_precision);
  SB_REQUIRE(p->quantize_bits == 0 || (p->quantize_bits >= 8 && p->quantize_bits <= 23),
             SB_ERR_INVALID_ARG, "quantize_bits must be 0 or in [8, 23]");
  SB_REQUIRE(p->tree_method == SB_TREE_HIST || p->tree_method == SB_TREE_APPROX, SB_ERR_INVALID_ARG,
             "unknown tree_method %d", p->tree_method);
  // Limits of this backend (documented): depthwise trees up to depth 12 (the
  // level histograms are preallocated), lossguide up to 4096 leaves.
  if (p->grow_policy == SB_GROW_DEPTHWISE)
    SB_REQUIRE(p->max_depth >= 1 && p->max_depth <= 12, SB_ERR_UNSUPPORTED,
               "depthwise growth on the GPU supports max_depth in [1, 12], got %d", p->max_depth);
  if (p->grow_policy == SB_GROW_LOSSGUIDE)
    SB_REQUIRE(p->max_leaves <= 4096 && (p->max_leaves > 0 || p->max_depth <= 12), SB_ERR_UNSUPPORTED,
               "lossguide growth on the GPU supports at most 4096 leaves");
  return SB_OK;
}

int sb_ctx_create(int device, sb_ctx** out) {
  SB_REQUIRE(out != nullptr, SB_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    sb::set_error("no CUDA device available (%s); this library has no CPU fallback",
                  cudaGetErrorString(e));
    return SB_ERR_NO_DEVICE;
  }
  SB_REQUIRE(device >= 0 && device < count, SB_ERR_INVALID_ARG, "device %d out of range", device);
  cudaDeviceProp prop;
  SB_CUDA(cudaGetDeviceProperties(&prop, device));
  SB_REQUIRE(prop.major == 10 && prop.minor == 0, SB_ERR_NO_DEVICE,
             "device %d is sm_%d%d; this library is built for sm_100a (B200) only", device,
             prop.major, prop.minor);
  SB_CUDA(cudaSetDevice(device));
  sb_ctx* c = new sb_ctx;
  c->device = device;
  c->num_sms = prop.multiProcessorCount;
  c->smem_optin = prop.sharedMemPerBlockOptin;
  c->smem_per_sm = prop.sharedMemPerMultiprocessor;
  cudaError_t se = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (se != cudaSuccess) {
    delete c;
    return sb::cuda_status(se, "cudaStreamCreate", __FILE__, __LINE__);
  }
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;  // keep freed blocks cached in the pool
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  cudaGetLastError();
  *out = c;
  return SB_OK;
}

int sb_ctx_destroy(sb_ctx* ctx) {
  if (!ctx) return SB_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return SB_OK;
}

int sb_ctx_synchronize(sb_ctx* ctx) {
  SB_REQUIRE(ctx != nullptr, SB_ERR_INVALID_ARG, "ctx is NULL");
  SB_CUDA(cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

void* sb_ctx_stream(sb_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }
uint64_t sb_ctx_launch_count(const sb_ctx* ctx) { return ctx ? ctx->launches.load() : 0; }

// ------------------------------------------------------------------ model
int sb_model_create(sb_ctx* ctx, const sb_model_view* v, sb_model** out) {
  SB_REQUIRE(ctx && v && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(v->n_trees >= 0, SB_ERR_INVALID_ARG, "negative n_trees");
  SB_REQUIRE(v->n_trees == 0 || (v->tree_node_offset && v->nodes), SB_ERR_INVALID_ARG,
             "model view without nodes");
  sb_model* m = new sb_model;
  m->ctx = ctx;
  m->base_score = v->base_score;
  m->num_class = v->num_class;
  m->n_features = v->n_features;
  m->objective = v->objective;
  m->trees.resize(v->n_trees);
  m->weights.resize(v->n_trees, 1.0f);
  for (int t = 0; t < v->n_trees; ++t) {
    int64_t b = v->tree_node_offset[t], e = v->tree_node_offset[t + 1];
    if (e <= b) {
      delete m;
      sb::set_error("tree %d has no nodes", t);
      return SB_ERR_INVALID_ARG;
    }
    m->trees[t].nodes.assign(v->nodes + b, v->nodes + e);
    if (v->categories && v->tree_cat_offset)
      m->trees[t].cats.assign(v->categories + v->tree_cat_offset[t],
                              v->categories + v->tree_cat_offset[t + 1]);
    if (v->tree_weights) m->weights[t] = v->tree_weights[t];
    // structural checks: children in range, no cycles (children > parent)
    int64_t nn = e - b;
    for (int64_t i = 0; i < nn; ++i) {
      const sb_node& nd = m->trees[t].nodes[i];
      bool leaf = nd.left < 0;
      if (!leaf && (nd.left <= i || nd.right <= i || nd.left >= nn || nd.right >= nn ||
                    (int)nd.split_feature >= v->n_features ||
                    (nd.is_categorical && nd.cat_end > m->trees[t].cats.size()))) {
        sb::set_error("tree %d node %lld is malformed", t, (long long)i);
        delete m;
        return SB_ERR_INVALID_ARG;
      }
    }
  }
  *out = m;
  return SB_OK;
}

int sb_model_destroy(sb_model* m) {
  delete m;
  return SB_OK;
}

int sb_model_export_sizes(const sb_model* m, int32_t* n_trees, int64_t* n_nodes, int64_t* n_cats) {
  SB_REQUIRE(m != nullptr, SB_ERR_INVALID_ARG, "model is NULL");
  int64_t nn = 0, nc = 0;
  for (auto& t : m->trees) {
    nn += (int64_t)t.nodes.size();
    nc += (int64_t)t.cats.size();
  }
  if (n_trees) *n_trees = (int32_t)m->trees.size();
  if (n_nodes) *n_nodes = nn;
  if (n_cats) *n_cats = nc;
  return SB_OK;
}

int sb_model_export(const sb_model* m, int64_t* node_off, sb_node* nodes, int64_t* cat_off,
                    uint32_t* cats, float* weights) {
  SB_REQUIRE(m != nullptr, SB_ERR_INVALID_ARG, "model is NULL");
  int64_t no = 0, co = 0;
  for (size_t t = 0; t < m->trees.size(); ++t) {
    const auto& tr = m->trees[t];
    if (node_off) node_off[t] = no;
    if (cat_off) cat_off[t] = co;
    if (nodes) std::memcpy(nodes + no, tr.nodes.data(), tr.nodes.size() * sizeof(sb_node));
    if (cats && !tr.cats.empty()) std::memcpy(cats + co, tr.cats.data(), tr.cats.size() * 4);
    if (weights) weights[t] = m->weights[t];
    no += (int64_t)tr.nodes.size();
    co += (int64_t)tr.cats.size();
  }
  if (node_off) node_off[m->trees.size()] = no;
  if (cat_off) cat_off[m->trees.size()] = co;
  return SB_OK;
}

int sb_model_info(const sb_model* m, float* base_score, int32_t* num_class, int32_t* n_features,
                  int32_t* objective) {
  SB_REQUIRE(m != nullptr, SB_ERR_INVALID_ARG, "model is NULL");
  if (base_score) *base_score = m->base_score;
  if (num_class) *num_class = m->num_class;
  if (n_features) *n_features = m->n_features;
  if (objective) *objective = m->objective;
  return SB_OK;
}

}  // extern "C"
