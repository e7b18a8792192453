// flash_laststep.cu -- the last-time-step copies of the flash's Bulk arrays
// and of the skip cache: IsoT_FIM::UpdateLastTimeStep / ResetToLastTimeStep
// (src/OCPFluidMethod.cpp:2915-2960, 2859-2897) for the arrays FlashFIM and
// PassFlashValue write, and SkipStaAnaly::UpdateLastTimeStep /
// ResetToLastTimeStep (src/AcceleratePVT.cpp:122-138). The reference assigns
// one std::vector per array; here every array pair is one entry of a table
// and ONE kernel copies them all: tiles of 256 threads x 4 vectors, each
// block taking tiles grid-stride, each entry at the widest vector (16, 8, 4,
// 2 or 1 bytes) its source, destination and size allow. HBM-bound: it reads
// and writes each byte once.
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "ocp_flash.h"

namespace ocpf {
namespace {

constexpr int kCopyThreads = 256;
constexpr int kCopyItems   = 4;  // vectors per thread per tile
constexpr int kTileElems   = kCopyThreads * kCopyItems;

struct CopyTable {
    int32_t              n;
    int32_t              pad;
    const unsigned char* src[OCPF_COPY_MAX];
    unsigned char*       dst[OCPF_COPY_MAX];
    int64_t              elems[OCPF_COPY_MAX];           // vectors of the entry
    int64_t              first_tile[OCPF_COPY_MAX + 1];  // prefix over the entries' tiles
    int32_t              width[OCPF_COPY_MAX];           // bytes per vector
};
static_assert(sizeof(CopyTable) < 4096, "kernel parameter space");

template <class V>
__device__ __forceinline__ void copy_tile(const unsigned char* s, unsigned char* d, int64_t n, int64_t i0)
{
    const V* sv = reinterpret_cast<const V*>(s);
    V*       dv = reinterpret_cast<V*>(d);
    V        v[kCopyItems];
#pragma unroll
    for (int k = 0; k < kCopyItems; k++) {
        const int64_t i = i0 + (int64_t)k * kCopyThreads + threadIdx.x;
        if (i < n) v[k] = sv[i];
    }
#pragma unroll
    for (int k = 0; k < kCopyItems; k++) {
        const int64_t i = i0 + (int64_t)k * kCopyThreads + threadIdx.x;
        if (i < n) dv[i] = v[k];
    }
}

__global__ void __launch_bounds__(kCopyThreads) k_copy_pairs(const __grid_constant__ CopyTable t)
{
    const int64_t ntile = t.first_tile[t.n];
    int           e     = 0;
    for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        while (tile >= t.first_tile[e + 1]) e++;  // tiles only grow: the entry index too
        const int64_t i0 = (tile - t.first_tile[e]) * kTileElems;
        switch (t.width[e]) {
            case 16: copy_tile<uint4>(t.src[e], t.dst[e], t.elems[e], i0); break;
            case 8: copy_tile<uint2>(t.src[e], t.dst[e], t.elems[e], i0); break;
            case 4: copy_tile<uint32_t>(t.src[e], t.dst[e], t.elems[e], i0); break;
            case 2: copy_tile<uint16_t>(t.src[e], t.dst[e], t.elems[e], i0); break;
            default: copy_tile<uint8_t>(t.src[e], t.dst[e], t.elems[e], i0); break;
        }
    }
}

// Adds one pair to the table; OCPF_EINVAL for an overlap of source and
// destination or a negative size. Same pointers and empty arrays are no-ops.
int add_pair(CopyTable& t, void* dst, const void* src, int64_t bytes)
{
    if (bytes < 0) return OCPF_EINVAL;
    if (bytes == 0) return OCPF_OK;
    if (!dst || !src) return OCPF_EINVAL;
    if (dst == src) return OCPF_OK;
    const uintptr_t d = (uintptr_t)dst, s = (uintptr_t)src;
    if (d < s + (uintptr_t)bytes && s < d + (uintptr_t)bytes) return OCPF_EINVAL;
    if (t.n >= OCPF_COPY_MAX) return OCPF_EINVAL;
    const uintptr_t all = d | s | (uintptr_t)bytes;
    int             w   = 16;
    while (w > 1 && (all % (uintptr_t)w) != 0) w >>= 1;
    t.src[t.n]   = (const unsigned char*)src;
    t.dst[t.n]   = (unsigned char*)dst;
    t.width[t.n] = w;
    t.elems[t.n] = bytes / w;
    t.n++;
    return OCPF_OK;
}

int launch(CopyTable& t, cudaStream_t st)
{
    if (t.n == 0) return OCPF_OK;
    t.first_tile[0] = 0;
    for (int e = 0; e < t.n; e++) t.first_tile[e + 1] = t.first_tile[e] + (t.elems[e] + kTileElems - 1) / kTileElems;
    static int resident = 0;  // blocks the device holds at once
    if (!resident) {
        int dev = 0, sms = 0, per_sm = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_copy_pairs, kCopyThreads, 0) != cudaSuccess)
            return OCPF_ECUDA;
        resident = std::max(1, sms) * std::max(1, per_sm);
    }
    // one wave of resident blocks; more tiles go grid-stride
    const int64_t grid = std::min<int64_t>(t.first_tile[t.n], (int64_t)resident);
    k_copy_pairs<<<(unsigned)grid, kCopyThreads, 0, st>>>(t);
    return cudaGetLastError() == cudaSuccess ? OCPF_OK : OCPF_ECUDA;
}

// A field of the two structs: copied when both pointers are set; exactly one
// set is an error.
int add_field(CopyTable& t, void* dst, const void* src, int64_t bytes)
{
    if (!dst && !src) return OCPF_OK;
    if (!dst || !src) return OCPF_EINVAL;
    return add_pair(t, dst, src, bytes);
}

// Every array of the flash's last-step state, from (cur, skip) into (last,
// lskip) when `save`, the other way round otherwise.
int step_copy(int nc, int64_t ncell, const ocpf_fim_out* cur, const ocpf_skip* skip, const ocpf_fim_out* last,
              const ocpf_skip* lskip, void* stream, bool save)
{
    if (nc < 1 || nc > OCPF_MAX_NC || ncell < 0 || !cur || !last) return OCPF_EINVAL;
    if ((skip == nullptr) != (lskip == nullptr)) return OCPF_EINVAL;
    const int64_t n    = ncell;
    const int64_t ncom = nc + 1;
    const int64_t ncol = ncom + 1;
    const int64_t NP   = OCPF_NUM_PHASE;
    const int64_t d8 = 8 * n, u4 = 4 * n;
    CopyTable     t{};
    int           rc = OCPF_OK;
    auto f = [&](const void* a, const void* b, int64_t bytes) {
        if (rc != OCPF_OK) return;
        void*       dst = const_cast<void*>(save ? b : a);
        const void* src = save ? a : b;
        rc              = add_field(t, dst, src, bytes);
    };
    const ocpf_fim_out &c = *cur, &l = *last;
    f(c.phaseNum, l.phaseNum, u4);
    f(c.phaseExist, l.phaseExist, NP * u4);
    f(c.S, l.S, NP * d8);
    f(c.Nt, l.Nt, d8);
    f(c.vf, l.vf, d8);
    f(c.vfP, l.vfP, d8);
    f(c.vfi, l.vfi, ncom * d8);
    f(c.rho, l.rho, NP * d8);
    f(c.xi, l.xi, NP * d8);
    f(c.mu, l.mu, NP * d8);
    f(c.rhoP, l.rhoP, NP * d8);
    f(c.xiP, l.xiP, NP * d8);
    f(c.muP, l.muP, NP * d8);
    f(c.xij, l.xij, NP * ncom * d8);
    f(c.rhox, l.rhox, NP * ncom * d8);
    f(c.xix, l.xix, NP * ncom * d8);
    f(c.mux, l.mux, NP * ncom * d8);
    f(c.dSec_dPri, l.dSec_dPri, NP * ncol * ncol * d8);
    f(c.bRowSizedSdP, l.bRowSizedSdP, u4);
    f(c.pSderExist, l.pSderExist, NP * u4);
    f(c.pVnumCom, l.pVnumCom, NP * u4);
    f(c.nj, l.nj, NP * d8);
    f(c.ePEC, l.ePEC, d8);
    f(c.ftype, l.ftype, n);
    f(c.iters, l.iters, 5 * u4);
    f(c.status, l.status, 2 * n);
    if (skip) {
        const ocpf_skip &s = *skip, &ls = *lskip;
        f(s.flag, ls.flag, u4);
        f(s.minEig, ls.minEig, d8);
        f(s.P, ls.P, d8);
        f(s.T, ls.T, d8);
        f(s.z, ls.z, nc * d8);
    }
    if (rc != OCPF_OK) return rc;
    return launch(t, (cudaStream_t)stream);
}

}  // namespace
}  // namespace ocpf

extern "C" {

int ocpf_update_last_step(int nc, int64_t ncell, const ocpf_fim_out* cur, const ocpf_skip* skip,
                          const ocpf_fim_out* last, const ocpf_skip* last_skip, void* stream)
{
    return ocpf::step_copy(nc, ncell, cur, skip, last, last_skip, stream, true);
}

int ocpf_reset_to_last_step(int nc, int64_t ncell, const ocpf_fim_out* cur, const ocpf_skip* skip,
                            const ocpf_fim_out* last, const ocpf_skip* last_skip, void* stream)
{
    return ocpf::step_copy(nc, ncell, cur, skip, last, last_skip, stream, false);
}

int ocpf_copy_arrays(int narr, void* const* dst, const void* const* src, const int64_t* bytes, void* stream)
{
    if (narr < 0 || narr > OCPF_COPY_MAX) return OCPF_EINVAL;
    if (narr == 0) return OCPF_OK;
    if (!dst || !src || !bytes) return OCPF_EINVAL;
    ocpf::CopyTable t{};
    for (int i = 0; i < narr; i++) {
        const int rc = ocpf::add_pair(t, dst[i], src[i], bytes[i]);
        if (rc != OCPF_OK) return rc;
    }
    return ocpf::launch(t, (cudaStream_t)stream);
}

}  // extern "C"
