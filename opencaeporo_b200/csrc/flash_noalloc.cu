// flash_noalloc.cu -- ocpf_flash_fim_noalloc: the batched flash with its
// scratch in an array compiled into the library, for callers that cannot
// allocate device memory (see include/ocp_flash.h).
#include <cstring>
#include <mutex>

#include "flash_phased.cuh"

namespace ocpf {
// launch sequences of the batched form (flash_phased_ncN.cu)
cudaError_t launch_phased_nc3(const FluidConst& F, const PhasedArgs& a, const LaunchTune& t, cudaStream_t st,
                              const cudaEvent_t* marks, const SideStreams* side);
cudaError_t launch_phased_nc6(const FluidConst& F, const PhasedArgs& a, const LaunchTune& t, cudaStream_t st,
                              const cudaEvent_t* marks, const SideStreams* side);
cudaError_t launch_phased_nc9(const FluidConst& F, const PhasedArgs& a, const LaunchTune& t, cudaStream_t st,
                              const cudaEvent_t* marks, const SideStreams* side);
cudaError_t launch_phased_nc12(const FluidConst& F, const PhasedArgs& a, const LaunchTune& t, cudaStream_t st,
                              const cudaEvent_t* marks, const SideStreams* side);
// context accessors (flash_api.cu)
const FluidConst* ctx_fluid_const(const ocpf_ctx* c);
int               ctx_device(const ocpf_ctx* c);
bool ctx_fim_args_ok(const ocpf_ctx* c, const ocpf_fim_in* in, const ocpf_skip* sk, const ocpf_fim_out* o);
}  // namespace ocpf

namespace {

using namespace ocpf;

constexpr int64_t kMaxCells = OCPF_NOALLOC_MAX_CELLS;
// Scratch per cell for the largest component count the batched kernels are
// built for (12): phase state doubles and ints, plus one slot in each list.
constexpr size_t kPerCell = 8 * (size_t)SF<12>::COUNT + 4 * (size_t)IF_COUNT + 4 * (size_t)L_COUNT;
constexpr size_t kBytes   = kPerCell * (size_t)kMaxCells + 8 * (size_t)L_COUNT + 256;

constexpr int kMaxDevices = 64;
std::mutex    g_mu;
void*         g_addr[kMaxDevices] = {};  // device address of the scratch, per device

}  // namespace

// The scratch of every ocpf_flash_fim_noalloc call on a device. In host code
// this name is only a handle for cudaGetSymbolAddress, never a device address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kBytes];

extern "C" int ocpf_flash_fim_noalloc(ocpf_ctx* ctx, int64_t ncell, const ocpf_fim_in* in, ocpf_skip* sk,
                                      ocpf_fim_out* out, void* stream)
{
    if (!ctx || ncell < 0) return OCPF_EINVAL;
    if (ncell > kMaxCells) return OCPF_ERANGE;
    if (ncell == 0) return OCPF_OK;
    if (!ctx_fim_args_ok(ctx, in, sk, out)) return OCPF_EINVAL;
    const FluidConst& F = *ctx_fluid_const(ctx);
    int               nd;
    cudaError_t (*launch)(const FluidConst&, const PhasedArgs&, const LaunchTune&, cudaStream_t, const cudaEvent_t*,
                          const SideStreams*);
    switch (F.nc) {
        case 3: launch = launch_phased_nc3, nd = SF<3>::COUNT; break;
        case 6: launch = launch_phased_nc6, nd = SF<6>::COUNT; break;
        case 9: launch = launch_phased_nc9, nd = SF<9>::COUNT; break;
        case 12: launch = launch_phased_nc12, nd = SF<12>::COUNT; break;
        default: return OCPF_EUNSUPPORTED;
    }
    const int dev = ctx_device(ctx);
    if (dev < 0 || dev >= kMaxDevices) return OCPF_EUNSUPPORTED;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return OCPF_ECUDA;

    // Once per device, with that device current: the array's device address.
    void* base = nullptr;
    int   rc   = OCPF_OK;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_addr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) == cudaSuccess && p)
                g_addr[dev] = p;
            else
                rc = OCPF_ECUDA;
        }
        base = g_addr[dev];
    }
    if (rc == OCPF_OK) {
        // same layout as the context scratch of ocpf_flash_fim, stride kMaxCells
        PhasedArgs a;
        std::memset(&a, 0, sizeof(a));  // every field not set below is zero / null
        a.tail   = FlashTail{FM_FIM, nullptr, nullptr, nullptr};
        a.count  = ncell;
        a.stride = ncell;
        a.in     = *in;
        a.sk     = sk ? *sk : ocpf_skip{};
        a.out    = *out;
        a.opts   = 0;
        a.mlp    = nullptr;
        a.S.cap  = kMaxCells;
        a.S.d    = (double*)base;
        a.S.i    = (int32_t*)(a.S.d + (size_t)nd * kMaxCells);
        a.L.cap  = kMaxCells;
        a.L.items = a.S.i + (size_t)IF_COUNT * kMaxCells;
        a.L.ctr   = (uint32_t*)(a.L.items + (size_t)L_COUNT * kMaxCells);
        // the launch sequence zeroes the list counters on the stream first;
        // every other scratch field a cell reads is written for it earlier in
        // the same call
        if (launch(F, a, kDefaultTune, (cudaStream_t)stream, nullptr, nullptr) != cudaSuccess) rc = OCPF_ECUDA;
    }
    if (prev != dev) cudaSetDevice(prev);
    return rc;
}
