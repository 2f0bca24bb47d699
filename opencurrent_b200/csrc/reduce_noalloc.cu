// ocu_grid_reduce_noalloc: the grid reduction with its scratch in a static device array.
//
// Some callers cannot allocate device memory at the point where they need a norm: code that
// runs while another framework's caching allocator owns the whole device, hosts that reserve
// all GPU memory up front and forbid later allocations, and latency-critical loops that must
// not touch the allocator.  ocu_grid_reduce takes its scratch from cudaMallocAsync; this entry
// point instead uses one fixed array that lives in the library's device image, so it performs
// no allocation at all.
//
// Limits and sharing rules (also stated in include/ocu_b200.h):
//   - the array holds the partials of at most OCU_REDUCE_NOALLOC_MAX_BLOCKS blocks of 256 rows,
//     i.e. grids with nx*ny <= 256 * OCU_REDUCE_NOALLOC_MAX_BLOCKS; larger grids are rejected
//     with OCU_ERR_INVALID_VALUE before anything is enqueued;
//   - every GPU that loads the library holds the array until the process exits;
//   - all calls on a device share the one array and it keeps the last call's contents, so each
//     call clears the parts that must start at zero; calls whose work overlaps on the GPU
//     (different streams, or different host threads, without ordering between them) race on
//     the array and must be serialised by the caller;
//   - the first call on a device looks the array's address up with cudaGetSymbolAddress while
//     that device is current; make that first call before any stream capture begins.
#include <mutex>

#include "ocu_internal.h"

namespace {

// [0, 8): result (double) | [64, 68): ticket counter | [128, ...): block partials (<= 8 B each)
constexpr size_t kResultOffset = 0;
constexpr size_t kCounterOffset = 64;
constexpr size_t kScratchBytes = 128 + 8 * (size_t)OCU_REDUCE_NOALLOC_MAX_BLOCKS;

__device__ __align__(256) unsigned char g_reduce_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {nullptr};

// Once per device, with that device current: the array's device address.  In host code the
// symbol g_reduce_scratch is only a host-side stand-in; passing it to a kernel would not
// reach the device array, so kernels receive this looked-up address instead.
ocu_status scratch_address(void **out) {
  int dev = -1;
  OCU_TRY(ocub::check_cuda(cudaGetDevice(&dev), "ocu_grid_reduce_noalloc: cudaGetDevice"));
  if (dev < 0 || dev >= kMaxDevices)
    return ocub::fail(OCU_ERR_UNSUPPORTED, "[ERROR] ocu_grid_reduce_noalloc - device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    OCU_TRY(ocub::check_cuda(cudaGetSymbolAddress(&p, g_reduce_scratch),
                             "ocu_grid_reduce_noalloc: cudaGetSymbolAddress"));
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return OCU_OK;
}

}  // namespace

extern "C" ocu_status ocu_grid_reduce_noalloc(const ocu_grid *g, ocu_reduce_op op, double *result, ocu_stream s) {
  using namespace ocub;
  if (!g || !result) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_grid_reduce_noalloc - null argument");
  if (op < OCU_REDUCE_MAXABS || op > OCU_REDUCE_CHECKNAN)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_grid_reduce_noalloc - bad op");
  const long long nrows = (long long)g->L.nx * g->L.ny;
  const long long blocks = (nrows + 255) / 256;
  if (nrows < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] ocu_grid_reduce_noalloc - empty grid");
  if (blocks > OCU_REDUCE_NOALLOC_MAX_BLOCKS)
    return fail(OCU_ERR_INVALID_VALUE,
                "[ERROR] ocu_grid_reduce_noalloc - grid has nx*ny = %lld rows; the static scratch holds at most "
                "%lld (use ocu_grid_reduce)",
                nrows, 256LL * OCU_REDUCE_NOALLOC_MAX_BLOCKS);
  void *base = nullptr;
  OCU_TRY(scratch_address(&base));
  cudaStream_t st = (cudaStream_t)s;
  char *p = static_cast<char *>(base);
  // the array keeps the previous call's contents: zero the result and the ticket counter
  OCU_TRY(check_cuda(cudaMemsetAsync(p, 0, 128, st), "ocu_grid_reduce_noalloc: clear scratch"));
  double *d_res = reinterpret_cast<double *>(p + kResultOffset);
  void *counter_and_partials = p + kCounterOffset;  // launch_reduce: counter at +0, partials at +64
  if (g->dtype == OCU_F64)
    OCU_TRY(launch_reduce<double>(origin<double>(g), g->L, op, counter_and_partials, d_res, st));
  else
    OCU_TRY(launch_reduce<float>(origin<float>(g), g->L, op, counter_and_partials, d_res, st));
  double h = 0;
  OCU_TRY(check_cuda(cudaMemcpyAsync(&h, d_res, sizeof(double), cudaMemcpyDeviceToHost, st),
                     "ocu_grid_reduce_noalloc: result readback"));
  OCU_TRY(check_cuda(cudaStreamSynchronize(st), "ocu_grid_reduce_noalloc"));
  *result = h;
  return OCU_OK;
}
