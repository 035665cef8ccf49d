// das_noalloc.cu -- batched DAS for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a process whose device memory belongs
// to another framework's pool or a fixed budget set at start-up, firmware-like
// real-time pipelines that forbid allocation after initialisation, or code that
// runs while allocation would deadlock or fragment a shared GPU. For them this
// file offers one entry point, dream_das_batch_run_noalloc, that beamforms a
// batch of frames with the persistent batch kernel without allocating
// anything: the work queue counter, the frame table and the tile list live in
// a file-scope device array of NOALLOC_SCRATCH_BYTES (4 MiB). Every GPU that
// loads this library holds that array until the process exits. The caller
// still provides every input and output buffer.
//
// The array is shared by all calls and keeps the last call's contents; the
// queue counter is cleared on the stream before each launch. Calls that
// overlap on the GPU (different streams, or different host threads) race on
// the array and must not be issued; calls on one stream are ordered.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/dream_das.h"
#include "das_fast.h"
#include "das_kernels.h"

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(4) << 20;
constexpr size_t CTR_BYTES = 256;
constexpr int MAX_DEVICES = 64;

// Device scratch. In host code this name is only a stand-in for the symbol:
// the device address comes from cudaGetSymbolAddress (noalloc_scratch_ptr).
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Host staging area for the frame table and tile list (no heap allocation).
alignas(256) static unsigned char g_host_stage[NOALLOC_SCRATCH_BYTES];
static void *g_dev_scratch[MAX_DEVICES];
static std::mutex g_mu;

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

// Once per device, with that device current: the scratch array's device address.
cudaError_t noalloc_scratch_ptr(int device, void **ptr) {
  if (g_dev_scratch[device] == nullptr) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_dev_scratch[device] = p;
  }
  *ptr = g_dev_scratch[device];
  return cudaSuccess;
}

}  // namespace

extern "C" int dream_das_batch_run_noalloc(const dream_das_frame *fr, int n_frames, int precision, int device,
                                           unsigned long long *d_oob, void *stream) {
  DREAM_API_TRY
  using namespace dream;
  if ((fr == nullptr && n_frames > 0) || n_frames < 0) return set_last_error(DREAM_ERR_ARGUMENT, "NULL argument");
  if (precision != DREAM_PREC_F32_STORE && precision != DREAM_PREC_BF16_STORE)
    return set_last_error(DREAM_ERR_UNSUPPORTED, "batches use F32_STORE or BF16_STORE");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  if (device < 0 || device >= ndev || device >= MAX_DEVICES)
    return set_last_error(DREAM_ERR_ARGUMENT, "invalid CUDA device ordinal");
  // The frame table and tile list are staged in a host array that every call
  // rewrites, and copied from there on the stream; a graph captured from this
  // call would re-read that array when replayed. So a stream that is being
  // captured is refused.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if ((e = cudaStreamIsCapturing((cudaStream_t)stream, &cap)) != cudaSuccess)
    return set_last_error(DREAM_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
  if (cap != cudaStreamCaptureStatusNone)
    return set_last_error(DREAM_ERR_UNSUPPORTED,
                          "dream_das_batch_run_noalloc cannot run on a stream that is being captured: it copies "
                          "its frame table from a host array that every call rewrites");
  std::lock_guard<std::mutex> lk(g_mu);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, "cudaSetDevice failed");
  struct Restore {
    int prev, dev;
    ~Restore() {
      if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
  } restore{prev, device};

  // ---- frame table in the host stage, then the tile list after it ----
  const size_t frames_off = CTR_BYTES;
  const size_t frames_bytes = round256((size_t)n_frames * sizeof(FastParams));
  const size_t order_off = frames_off + frames_bytes;  // host only: frame order
  const size_t order_bytes = round256((size_t)n_frames * sizeof(int));
  if (frames_off + frames_bytes + order_bytes > NOALLOC_SCRATCH_BYTES)
    return set_last_error(DREAM_ERR_ARGUMENT, "batch too large for the allocation-free entry point: " +
                                                  std::to_string(n_frames) + " frames need more than its 4 MiB scratch");
  FastParams *T = reinterpret_cast<FastParams *>(g_host_stage + frames_off);
  int *order = reinterpret_cast<int *>(g_host_stage + order_off);
  size_t smem = 1024;
  for (int f = 0; f < n_frames; f++) {
    FastParams &F = T[f];
    const int r = batch_frame_params(fr[f], F);
    if (r) return r;
    F.oob = d_oob;
    smem = std::max(smem, fast_smem_bytes(F, 128));
    order[f] = f;
  }
  if (smem > 220 * 1024)
    return set_last_error(DREAM_ERR_UNSUPPORTED, "a frame has too many outer elements for the batch kernel");
  // largest per-tile cost first (as dream_das_batch_create)
  std::stable_sort(order, order + n_frames, [&](int a, int b) {
    return (double)T[a].Nt * T[a].Nr > (double)T[b].Nt * T[b].Nr;
  });
  const size_t items_off = frames_off + frames_bytes;  // on the device the tile list follows the frames
  int4 *items = reinterpret_cast<int4 *>(g_host_stage + order_off + order_bytes);
  const size_t items_cap = (NOALLOC_SCRATCH_BYTES - (order_off + order_bytes)) / sizeof(int4);
  const size_t dev_items_cap = (NOALLOC_SCRATCH_BYTES - items_off) / sizeof(int4);
  size_t n_items = 0;
  for (int q = 0; q < n_frames; q++) {
    const FastParams &F = T[order[q]];
    if (F.No == 0 || F.K == 0) continue;
    const int64_t tf = (F.n_fast + F.tile_f - 1) / F.tile_f, ts = (F.n_slow + F.tile_s - 1) / F.tile_s;
    if ((double)tf * ts + n_items > (double)std::min(items_cap, dev_items_cap))
      return set_last_error(DREAM_ERR_ARGUMENT,
                            "batch too large for the allocation-free entry point: more than " +
                                std::to_string(std::min(items_cap, dev_items_cap)) + " tiles in its 4 MiB scratch");
    for (int64_t s = 0; s < ts; s++)
      for (int64_t t = 0; t < tf; t++) items[n_items++] = make_int4(order[q], (int)t, (int)s, 0);
  }

  // ---- device scratch: set up once per device, then one copy and the launch ----
  void *dev = nullptr;
  if ((e = noalloc_scratch_ptr(device, &dev)) != cudaSuccess)
    return set_last_error(DREAM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  unsigned char *base = static_cast<unsigned char *>(dev);
  cudaStream_t st = (cudaStream_t)stream;
  if (n_frames > 0 &&
      (e = cudaMemcpyAsync(base + frames_off, T, (size_t)n_frames * sizeof(FastParams), cudaMemcpyHostToDevice, st)) !=
          cudaSuccess)
    return set_last_error(DREAM_ERR_CUDA, std::string("frame table copy: ") + cudaGetErrorString(e));
  if (n_items > 0 &&
      (e = cudaMemcpyAsync(base + items_off, items, n_items * sizeof(int4), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return set_last_error(DREAM_ERR_CUDA, std::string("tile list copy: ") + cudaGetErrorString(e));
  const bool bf16 = precision == DREAM_PREC_BF16_STORE;
  const int per_sm = batch_prepare(smem, bf16);
  if (per_sm <= 0) return set_last_error(DREAM_ERR_CUDA, "batch kernel does not fit on an SM");
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int grid = (int)std::min<int64_t>((int64_t)sms * per_sm, std::max<int64_t>(1, (int64_t)n_items));
  e = launch_batch(reinterpret_cast<const FastParams *>(base + frames_off), reinterpret_cast<const int4 *>(base + items_off),
                   (int)n_items, reinterpret_cast<int *>(base), smem, bf16, grid, st);
  if (e != cudaSuccess) return set_last_error(DREAM_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
  return 0;
  DREAM_API_CATCH
}
