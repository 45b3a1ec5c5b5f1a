// vfrb_dedisperse_noalloc: dedispersion + per-DM statistics with the
// statistics scratch in a fixed device array instead of caller memory.
//
// Who needs it: callers that may not allocate device memory after start-up
// (a real-time loop whose allocator is frozen, a host language whose binding
// cannot hand out device buffers, code running between graph-capture
// boundaries) but still want the per-DM mean/sigma/peak/FRB flag that
// vfrb_dedisperse computes.  That computation needs per-(time block, DM)
// partial sums; vfrb_dedisperse takes them in caller-provided `workspace`,
// this entry point takes them in g_dd_scratch below, so it calls neither
// cudaMalloc nor cudaFree nor any allocating library.
//
// Limit: the partials need vfrb_dedisperse_workspace_bytes(plan, nt_out) =
// ndm * ceil(nt_out / 256) * 24 bytes, and g_dd_scratch holds
// VFRB_NOALLOC_SCRATCH_BYTES (4 MiB), e.g. 2048 DMs x 21,760 samples.
// Larger requests return VFRB_ERR_ARG before anything is launched.
#include <mutex>

#include "vfrb_common.cuh"

namespace vfrb {
size_t dedisperse_workspace_bytes_plan(const vfrb_ddplan* pl, long long nt_out);
int launch_dedisperse_plan(const vfrb_ddplan* pl, const vfrb_dd_args& a, cudaStream_t s);
}  // namespace vfrb

namespace {

constexpr size_t kScratchBytes = VFRB_NOALLOC_SCRATCH_BYTES;
static_assert(kScratchBytes % 256 == 0, "scratch is a whole number of 256-byte lines");

// One copy per device (each device that loads the module gets its own).  It
// holds only partial sums that every call writes in full before it reads
// them, so nothing in it has to start at zero.
static __device__ __align__(256) unsigned char g_dd_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
struct ScratchEntry {
  void* ctx;  // CUDA context the address belongs to
  void* ptr;
};
ScratchEntry g_scratch[kMaxDevices] = {};

// cuCtxGetCurrent through the runtime's driver entry point (no link against
// libcuda); null when the driver does not offer it.
using CtxGetCurrentFn = int (*)(void**);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (CtxGetCurrentFn) nullptr;
    }
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  return fn;
}

// Device address of g_dd_scratch in the current device's current context.
// It is looked up once per device and context (the lookup may load the
// module, so make the first call on a device before any stream capture) and
// looked up again when the device's context changes (another context made
// current, or the primary context re-created after cudaDeviceReset).
int scratch_for_current_device(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return VFRB_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return VFRB_ERR_UNSUPPORTED;
  // Before the runtime has bound a context to this thread there is none to
  // key on; the address is then looked up (which binds the primary context)
  // and keyed on the next call.
  void* ctx = nullptr;
  CtxGetCurrentFn cur = ctx_get_current();
  const bool have_ctx = cur && cur(&ctx) == 0 && ctx;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  ScratchEntry& ent = g_scratch[dev];
  if (!have_ctx || !ent.ptr || ent.ctx != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_dd_scratch);
    if (e != cudaSuccess || !p) return VFRB_ERR_CUDA;
    ent.ptr = p;
    ent.ctx = have_ctx ? ctx : nullptr;
  }
  *out = ent.ptr;
  return VFRB_OK;
}

}  // namespace

extern "C" size_t vfrb_dedisperse_noalloc_scratch_bytes(void) { return kScratchBytes; }

extern "C" int vfrb_dedisperse_noalloc(const vfrb_ddplan* plan, const vfrb_dd_args* a, void* stream) {
  if (!plan || !a) return VFRB_ERR_ARG;
  const bool want_stats = a->ave || a->sigma || a->peak || a->frb || a->argmax;
  vfrb_dd_args b = *a;
  b.workspace = nullptr;
  b.workspace_bytes = 0;
  if (want_stats && a->nt_out > 0) {
    // size check first: nothing is set up or launched for a request that
    // does not fit the fixed scratch
    if (vfrb::dedisperse_workspace_bytes_plan(plan, a->nt_out) > kScratchBytes) return VFRB_ERR_ARG;
    const int st = scratch_for_current_device(&b.workspace);
    if (st != VFRB_OK) return st;
    b.workspace_bytes = kScratchBytes;
  }
  return vfrb::launch_dedisperse_plan(plan, b, (cudaStream_t)stream);
}
