// sb_static.cu — sb_hist_build_static: the FP32 histogram build of one node
// into caller-owned device buffers, with no device memory allocated by the
// library.
//
// Its working memory (the node histogram with the per-feature missing bins,
// the one-item work list and the feature tiles) lives in one file-scope
// device array, SB_STATIC_SCRATCH_BYTES long, whose address is looked up once
// per device. Every call on every context of a device uses the same array.
#include <mutex>

#include "sb_internal.cuh"

namespace sb {

static __device__ __align__(256) unsigned char g_static_scratch[SB_STATIC_SCRATCH_BYTES];

namespace {

constexpr int STATIC_MAX_DEVICES = 64;
std::mutex g_static_mu;
unsigned char* g_static_ptr[STATIC_MAX_DEVICES];  // device address of g_static_scratch, per device

// The scratch address on `device` (the current device). The first call on a
// device resolves it with cudaGetSymbolAddress.
int static_scratch(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_static_mu);
  SB_REQUIRE(device >= 0 && device < STATIC_MAX_DEVICES, SB_ERR_UNSUPPORTED,
             "sb_hist_build_static: device ordinal %d is above %d", device, STATIC_MAX_DEVICES - 1);
  if (!g_static_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error("sb_hist_build_static: cudaGetSymbolAddress of the scratch array failed on device %d: %s",
                device, cudaGetErrorString(e));
      return SB_ERR_CUDA;
    }
    g_static_ptr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_static_ptr[device];
  return SB_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Counts row ids that are not below n (the caller's rows are not read on the host).
__global__ void k_count_bad_rows(const uint32_t* __restrict__ rows, size_t m, size_t n,
                                 unsigned int* __restrict__ bad) {
  unsigned int c = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
    c += rows[i] >= n ? 1u : 0u;
  if (c) atomicAdd(bad, c);
}

}  // namespace
}  // namespace sb

extern "C" {

int sb_hist_build_static(sb_ctx* ctx, const sb_ghist* g, const uint32_t* d_rows, size_t m,
                         const sb_gradpair* d_gpair, size_t n, sb_gradstats* d_out, size_t total_bins) {
  using namespace sb;
  SB_REQUIRE(ctx && g && d_gpair && d_out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_SAME_DEVICE(ctx, g);
  SB_REQUIRE(m == 0 || d_rows, SB_ERR_INVALID_ARG, "d_rows is NULL");
  SB_REQUIRE(total_bins == g->total_bins, SB_ERR_DIMENSION,
             "dimension mismatch: out length expected %zu, got %zu", g->total_bins, total_bins);
  SB_REQUIRE(n == g->n, SB_ERR_DIMENSION, "dimension mismatch: gpair length expected %zu, got %zu",
             g->n, n);
  SB_REQUIRE(m <= 0xFFFFFFFFull, SB_ERR_INVALID_ARG, "more than 2^32 - 1 rows");

  // scratch layout: node histogram | work item | prefix | item count | bad-row count | tiles
  const size_t HB = g->total_bins + g->F;
  const size_t off_item = align256(HB * sizeof(double2));
  const size_t off_prefix = off_item + align256(sizeof(HistItem));
  const size_t off_count = off_prefix + align256(2 * sizeof(uint64_t));
  const size_t off_bad = off_count + align256(sizeof(int));
  const size_t off_tiles = off_bad + align256(sizeof(unsigned int));
  const size_t need = off_tiles + g->tiles.size() * sizeof(FeatureTile);
  SB_REQUIRE(need <= SB_STATIC_SCRATCH_BYTES, SB_ERR_UNSUPPORTED,
             "sb_hist_build_static: %zu bins need %zu bytes of scratch, above the %zu-byte limit "
             "(SB_STATIC_SCRATCH_BYTES); use sb_hist_build",
             HB, need, (size_t)SB_STATIC_SCRATCH_BYTES);

  SB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  // the call copies its small tables from host memory and waits for its
  // result, so it cannot be recorded into a graph
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  SB_CUDA(cudaStreamIsCapturing(st, &cap));
  SB_REQUIRE(cap == cudaStreamCaptureStatusNone, SB_ERR_UNSUPPORTED,
             "sb_hist_build_static cannot run while the context's stream is being captured");
  unsigned char* base = nullptr;
  SB_TRY(static_scratch(ctx->device, &base));
  double2* hist = reinterpret_cast<double2*>(base);
  HistItem* d_item = reinterpret_cast<HistItem*>(base + off_item);
  uint64_t* d_prefix = reinterpret_cast<uint64_t*>(base + off_prefix);
  int* d_count = reinterpret_cast<int*>(base + off_count);
  unsigned int* d_bad = reinterpret_cast<unsigned int*>(base + off_bad);
  FeatureTile* d_tiles = reinterpret_cast<FeatureTile*>(base + off_tiles);

  // the row ids must index the gradient and bin arrays
  if (m) {
    SB_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(unsigned int), st));
    const unsigned blocks = (unsigned)std::min<size_t>((m + 255) / 256, (size_t)ctx->num_sms * 4);
    SB_LAUNCH(ctx, k_count_bad_rows, blocks, 256, 0, d_rows, m, n, d_bad);
    unsigned int bad = 0;
    SB_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    SB_REQUIRE(bad == 0, SB_ERR_INVALID_ARG, "%u row ids are not below n_rows = %zu", bad, n);
  }

  // the histogram accumulates with atomics, so it starts at zero on every call
  SB_CUDA(cudaMemsetAsync(hist, 0, HB * sizeof(double2), st));
  HistItem it;
  it.rows = d_rows;
  it.begin = 0;
  it.end = (uint32_t)m;
  it.k = 0;
  it.root = 0;
  it.out = hist;
  it.total = nullptr;
  const uint64_t prefix[2] = {0, (uint64_t)m};
  const int one = 1;
  SB_CUDA(cudaMemcpyAsync(d_item, &it, sizeof(it), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_prefix, prefix, sizeof(prefix), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_count, &one, sizeof(one), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_tiles, g->tiles.data(), g->tiles.size() * sizeof(FeatureTile),
                          cudaMemcpyHostToDevice, st));
  if (m) {
    HistLaunch L;
    L.g = g;
    L.gpair = d_gpair;
    L.fixed = 0;
    L.quant_bits = 16;
    L.items = d_item;
    L.prefix = d_prefix;
    L.count = d_count;
    L.max_items = 1;
    L.tiles = d_tiles;
    L.ntiles = (int)g->tiles.size();
    L.rows_done = nullptr;
    L.pool_mask = nullptr;
    SB_TRY(launch_hist(ctx, L));
  }
  // the present bins (global bin order); the missing bins stay in scratch
  SB_CUDA(cudaMemcpyAsync(d_out, hist, total_bins * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  SB_CUDA(cudaStreamSynchronize(st));
  return SB_OK;
}

}  // extern "C"
