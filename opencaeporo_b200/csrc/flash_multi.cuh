// flash_multi.cuh -- the batched flash of several PVT regions (fluids of
// different component counts) as ONE launch sequence: every step of the
// schedule in flash_phased.cuh is one kernel over all regions' cells.
//
//   * thread-per-item steps (set-up, verdicts, routing, finalize): block b
//     works for region b % n, with that region's share of the grid
//     (PhasedArgs::vpart / vparts);
//   * persistent steps (the substitution and Newton loops): each warp drains
//     the regions' lists one after another, starting at region (warp id mod
//     n), so the warps that finish a light fluid's list move on to a heavy
//     one's and no SM idles while any region has work;
//   * the component count is a compile-time constant inside each body: a
//     warp-uniform switch picks the body instantiated for its region's NC
//     (3, 6, 9 or 12), so per-cell state stays in registers.
//
// Each cell takes exactly the steps, in the same order and with the same
// expressions, as in the one-region sequence. No counterpart in the
// reference (its PVT regions are separate MixtureComp objects called cell by
// cell).
#pragma once

#include <type_traits>

#include "flash_learned.cuh"
#include "flash_mixed.cuh"
#include "flash_phased_kernels.cuh"

namespace ocpf {

constexpr int MULTI_MAX = 4;  // regions in one launch sequence

struct MultiFluid {
    FluidConst F[MULTI_MAX];
};
struct MultiArgs {
    int32_t    n;              // regions in this launch (1..MULTI_MAX)
    int32_t    nc[MULTI_MAX];  // their component counts
    PhasedArgs a[MULTI_MAX];   // their arguments (a[r].vpart = r, a[r].vparts = n)
};
static_assert(sizeof(MultiFluid) + sizeof(MultiArgs) + 64 < 32764, "kernel parameter space");

// Calls fn(std::integral_constant<int, NC>) for the region's component count.
template <class Fn>
__device__ __forceinline__ void with_nc(int nc, Fn&& fn)
{
    switch (nc) {
        case 3: fn(std::integral_constant<int, 3>{}); break;
        case 6: fn(std::integral_constant<int, 6>{}); break;
        case 9: fn(std::integral_constant<int, 9>{}); break;
        case 12: fn(std::integral_constant<int, 12>{}); break;
        default: break;
    }
}

// Thread-per-item (and warp-per-item) steps: the block's region. CALL is
// the body's call, written with NC_ (the region's component count), F_ (its
// fluid) and A_ (its arguments), in parentheses.
#define OCPF_MULTI_ITEMS(MF, M, CALL)                                  \
    {                                                                 \
        const int         r_ = (int)(blockIdx.x % (uint32_t)(M).n);   \
        const FluidConst& F_ = (MF).F[r_];                            \
        const PhasedArgs& A_ = (M).a[r_];                             \
        with_nc((M).nc[r_], [&](auto nc_) {                           \
            constexpr int NC_ = decltype(nc_)::value;                 \
            CALL;                                                     \
        });                                                           \
    }

// Persistent steps: every region's list in turn, from the warp's own.
#define OCPF_MULTI_PERSIST(MF, M, CALL)                                         \
    {                                                                          \
        const int w_ = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);    \
        for (int t_ = 0; t_ < (M).n; t_++) {                                   \
            const int         r_ = (w_ + t_) % (M).n;                          \
            const FluidConst& F_ = (MF).F[r_];                                 \
            const PhasedArgs& A_ = (M).a[r_];                                  \
            with_nc((M).nc[r_], [&](auto nc_) {                                \
                constexpr int NC_ = decltype(nc_)::value;                      \
                CALL;                                                          \
            });                                                                \
        }                                                                      \
    }

// Steps of the sequence. The kernels live in four units (for parallel
// builds: each holds every step's body for all four component counts);
// each unit's helper launches its steps and reports their occupancy.
enum MultiStep : int {
    MS_INIT, MS_S01_PREP, MS_S01_SSM, MS_S01_END, MS_STA_PREP, MS_LEARN,  // flash_multi_a.cu
    MS_STA_SSM, MS_STA_SSM32, MS_STA_VERDICT, MS_STA_NR,                  // flash_multi_b.cu
    MS_SP_PREP, MS_SP_SSM, MS_SP_NRINIT, MS_SP_NR,                        // flash_multi_c.cu
    MS_SLOW, MS_SLOW_THREAD, MS_FINALIZE, MS_FINALIZE_FIMN,               // flash_multi_d.cu
    MS_COUNT
};

#define OCPF_DECL_MULTI_UNIT(X)                                                                                \
    cudaError_t multi_step_##X(int s, const MultiFluid& MF, const MultiArgs& M, unsigned grid, int block,      \
                               size_t smem, cudaStream_t st, int i0, int i1, int i2, bool b0);                  \
    int         multi_occupancy_##X(int s);
OCPF_DECL_MULTI_UNIT(a)
OCPF_DECL_MULTI_UNIT(b)
OCPF_DECL_MULTI_UNIT(c)
OCPF_DECL_MULTI_UNIT(d)
#undef OCPF_DECL_MULTI_UNIT

// The whole launch sequence over the regions of M (flash_multi.cu). `count`
// of each region is its cell count.
cudaError_t launch_phased_multi(const MultiFluid& MF, const MultiArgs& M, const LaunchTune& t, cudaStream_t st);

}  // namespace ocpf
