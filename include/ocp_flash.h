/*
 * ocp_flash.h -- C ABI of the B200 compositional Peng-Robinson flash.
 *
 * One batched call replaces the reference's per-bulk flash loop
 *   IsoT_FIM::CalFlash (src/OCPFluidMethod.cpp:1108-1120):
 *     for n: flashCal[PVTNUM[n]]->FlashFIM(P[n], T[n], &Ni[n*nc], &S[n*np],
 *                                          phaseNum[n], &xij[n*np*nc], n);
 *            PassFlashValue(bk, n);            (src/OCPFluidMethod.cpp:1122-1187)
 * with MixtureComp::FlashFIM (src/MixtureComp.cpp:494-573, declared at
 * include/Mixture.hpp:106-112) evaluated for every cell on the GPU and the
 * results written straight into the caller's arrays, as PassFlashValue does.
 *
 * Conventions
 *   - nc hydrocarbon components; numCom = nc + 1 (water last); 3 phases
 *     (0 oil, 1 gas, 2 water), as in MixtureComp (src/MixtureComp.cpp:34-48).
 *   - FIELD units: psia, degF, ft3/lbmol, lbmol, lb/ft3, cP.
 *   - Every array pointer is a DEVICE pointer (ocpf_flash_fim_host excepted),
 *     laid out structure-of-arrays: field index slow, cell index fast, e.g.
 *     Ni[i*ncell + n], xij[(j*numCom + i)*ncell + n],
 *     dSec_dPri[(r*(numCom+1) + c)*ncell + n].
 *   - Outputs of phases that do not exist are left untouched (as
 *     PassFlashValue leaves them); S, phaseExist, the derivative-shape flags
 *     and the compact dSec_dPri rows are always written.
 *   - No call traps or aborts. Numerical trouble is reported per cell in
 *     `status` (OCPF_CELL_* bits); argument errors return OCPF_EINVAL.
 *   - Calls are stream-ordered and asynchronous on the given cudaStream_t
 *     (passed as void*; NULL = legacy default stream). A context may be used
 *     from one host thread at a time.
 */
#ifndef OCP_FLASH_H
#define OCP_FLASH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OCPF_MAX_NC 16
#define OCPF_NUM_PHASE 3

/* return codes */
#define OCPF_OK 0
#define OCPF_EINVAL 1       /* bad argument */
#define OCPF_ECUDA 2        /* a CUDA runtime call failed */
#define OCPF_ENOMEM 3       /* device allocation failed */
#define OCPF_EUNSUPPORTED 4 /* e.g. no sm_100 device */
#define OCPF_ERANGE 5       /* batch larger than OCPF_NOALLOC_MAX_CELLS (ocpf_flash_fim_noalloc) */

/* largest batch ocpf_flash_fim_noalloc accepts */
#define OCPF_NOALLOC_MAX_CELLS 4096
#define OCPF_KRPC_MAX_REGIONS 64 /* saturation regions (SATNUM values) per ocpf_krpc handle */

/* per-cell status bits (ocpf_fim_out.status) */
#define OCPF_CELL_SSMSTA_CAP 0x01  /* a stability SSM trial hit maxIt */
#define OCPF_CELL_NRSTA_FAIL 0x02  /* stability NR not converged */
#define OCPF_CELL_SSMSP_FAIL 0x04  /* split SSM not converged */
#define OCPF_CELL_NRSP_FAIL 0x08   /* split NR not converged */
#define OCPF_CELL_COLLAPSED 0x10   /* split collapsed to one phase (CheckSplit) */
#define OCPF_CELL_SINGULAR 0x20    /* a dense solve met a zero pivot */
#define OCPF_CELL_NONFINITE 0x40   /* a non-finite value reached an output */
#define OCPF_CELL_SPLIT_CAP 0x80   /* split restart loop bound reached */
#define OCPF_CELL_GUARD 0x100      /* internal control-flow bound reached (a bug if ever set) */

/* flash forms (all return the same outputs) */
#define OCPF_FORM_PLAIN 0   /* one thread per cell, FP64: the reference's algorithm as written */
#define OCPF_FORM_BATCHED 1 /* same FP64 arithmetic, persistent lane-refilling equilibrium
                               kernel + separate finalize kernel */
#define OCPF_FORM_MIXED 2   /* batched, successive substitution in FP32, FP64 Newton polish */
#define OCPF_FORM_FAST 3    /* mixed + learned initialiser where a model is loaded */

/* Fluid of one PVT region plus its solver controls: what MixtureComp's
 * constructor reads from ComponentParam (src/MixtureComp.cpp:28-165,
 * include/ParamReservoir.hpp:87-193) and the water PVTW row. */
typedef struct {
    int32_t nc;
    int32_t rr_maxit;     /* RR keyword */
    int32_t ssmsta_maxit; /* SSMSTA keyword */
    int32_t nrsta_maxit;  /* NRSTA keyword */
    int32_t ssmsp_maxit;  /* SSMSP keyword */
    int32_t nrsp_maxit;   /* NRSP keyword */
    int32_t use_skip;     /* SkipStaAnaly::ifUseSkip (include/AcceleratePVT.hpp:71) */
    int32_t pad0;
    double rr_tol, ssmsta_tol, ssmsta_eyt, nrsta_tol, ssmsp_tol, nrsp_tol;
    double Tc[OCPF_MAX_NC];     /* degR */
    double Pc[OCPF_MAX_NC];     /* psia */
    double Vc[OCPF_MAX_NC];     /* ft3/lbmol */
    double MW[OCPF_MAX_NC];
    double Acf[OCPF_MAX_NC];
    double OmegaA[OCPF_MAX_NC];
    double OmegaB[OCPF_MAX_NC];
    double Vshift[OCPF_MAX_NC]; /* dimensionless deck VSHIFT */
    double BIC[OCPF_MAX_NC * OCPF_MAX_NC]; /* nc*nc row-major, symmetric */
    double LBCcoef[5];          /* deck LBCCOEF (scaled by 10 inside, as the reference does) */
    double pvtw[5];             /* PVTW row: Pref, Bw, Cw, muw, Cvw */
    double std_rho_w;           /* lb/ft3 */
} ocpf_fluid;

/* Inputs of FlashFIM for every cell (device, SoA). xij and S are the
 * previous step's outputs (the Bulk arrays are passed in place), lastNP the
 * previous phase count with water included (Bulk::phaseNum). */
typedef struct {
    const double*   P;      /* [ncell] psia */
    const double*   T;      /* [ncell] degF */
    const double*   Ni;     /* [numCom][ncell] */
    const double*   S;      /* [3][ncell] */
    const uint32_t* lastNP; /* [ncell] */
    const double*   xij;    /* [3*numCom][ncell] */
} ocpf_fim_in;

/* Per-cell SkipStaAnaly cache (src/AcceleratePVT.cpp:135-233), read and
 * written in place; may be all-NULL when the fluid's use_skip is 0. */
typedef struct {
    uint32_t* flag;   /* [ncell] */
    double*   minEig; /* [ncell] */
    double*   P;      /* [ncell] */
    double*   T;      /* [ncell] degR (the flash's internal temperature) */
    double*   z;      /* [nc][ncell] */
} ocpf_skip;

/* Outputs (device, SoA), named as the Bulk arrays PassFlashValue fills.
 * Pointers marked optional may be NULL. */
typedef struct {
    uint32_t* phaseNum;     /* [ncell] phases present, water included */
    uint32_t* phaseExist;   /* [3][ncell] */
    double*   S;            /* [3][ncell] */
    double*   Nt;           /* [ncell] */
    double*   vf;           /* [ncell] */
    double*   vfP;          /* [ncell] */
    double*   vfi;          /* [numCom][ncell] */
    double*   rho;          /* [3][ncell] */
    double*   xi;           /* [3][ncell] */
    double*   mu;           /* [3][ncell] */
    double*   rhoP;         /* [3][ncell] */
    double*   xiP;          /* [3][ncell] */
    double*   muP;          /* [3][ncell] */
    double*   xij;          /* [3*numCom][ncell] (may alias ocpf_fim_in.xij) */
    double*   rhox;         /* [3*numCom][ncell] */
    double*   xix;          /* [3*numCom][ncell] */
    double*   mux;          /* [3*numCom][ncell] */
    double*   dSec_dPri;    /* [3*(numCom+1)^2][ncell], first bRowSizedSdP rows written */
    uint32_t* bRowSizedSdP; /* [ncell] */
    uint32_t* pSderExist;   /* [3][ncell] */
    uint32_t* pVnumCom;     /* [3][ncell] */
    /* optional diagnostics */
    double*   nj;           /* [3][ncell] phase moles */
    double*   ePEC;         /* [ncell] MixtureComp::ePEC */
    uint8_t*  ftype;        /* [ncell] flash type 0/1/2 */
    int32_t*  iters;        /* [5][ncell] SSMSTA, NRSTA, SSMSP, NRSP, RR iterations */
    uint16_t* status;       /* [ncell] OCPF_CELL_* bits */
} ocpf_fim_out;

/* FlashIMPEC's inputs (src/MixtureComp.cpp:444-450): no saturations. */
typedef struct {
    const double*   P;      /* [ncell] psia */
    const double*   T;      /* [ncell] degF */
    const double*   Ni;     /* [numCom][ncell] lbmol */
    const uint32_t* lastNP; /* [ncell] phase count of the last step (0: fresh) */
    const double*   xij;    /* [numPhase*numCom][ncell] last step's compositions */
} ocpf_impec_in;

/* The Bulk arrays IsoT_IMPEC::PassFlashValue fills (src/OCPFluidMethod.cpp:
 * 275-305), same layouts as ocpf_fim_out, plus the phase volumes vj. Outputs
 * of absent phases are left untouched, as there. The diagnostics may be
 * null. */
typedef struct {
    uint32_t* phaseNum;
    uint32_t* phaseExist;
    double*   S;
    double*   Nt;
    double*   vf;
    double*   vfP;
    double*   vfi;
    double*   vj;  /* [numPhase][ncell] ft3 */
    double*   rho;
    double*   xi;
    double*   mu;
    double*   xij;
    double*   ePEC;
    uint8_t*  ftype;
    int32_t*  iters;
    uint16_t* status;
} ocpf_impec_out;

/* The initial state InitFlashFIM / InitFlashIMPEC take per cell
 * (src/MixtureComp.cpp:261-267, :195-201, as IsoT_FIM::InitFlash and
 * IsoT_IMPEC::InitFlash pass the Bulk arrays, src/OCPFluidMethod.cpp:
 * 1095-1106, 251-262). The bubble-point pressure Pb the reference passes is
 * not used by the compositional flash and has no field. */
typedef struct {
    const double* P;     /* [ncell] psia */
    const double* T;     /* [ncell] degF */
    const double* S;     /* [numPhase][ncell] initial saturations; S_w (the last) is read */
    const double* Vpore; /* [ncell] pore volume (Bulk::rockVp), ft3 */
    const double* zi;    /* [numCom][ncell] initial mole fractions; the water entry is not read */
} ocpf_init_in;

typedef struct ocpf_ctx ocpf_ctx;

/* Library version string. */
const char* ocpf_version(void);

/* Human-readable text for a return code. */
const char* ocpf_status_string(int code);

/* Creates a flash context for one PVT region on the given CUDA device:
 * the counterpart of constructing MixtureComp(ParamReservoir, i)
 * (src/MixtureComp.cpp:28-165) and SetupOptionalFeatures
 * (src/MixtureComp.cpp:5128-5144). Derived constants are computed once here.
 * Returns OCPF_EINVAL for nc outside [2, OCPF_MAX_NC] or non-positive
 * critical properties. */
int ocpf_create(const ocpf_fluid* fluid, int device, ocpf_ctx** ctx);

/* Releases a context and every device buffer it owns. */
int ocpf_destroy(ocpf_ctx* ctx);

/* Batched MixtureComp::FlashFIM + PassFlashValue over ncell cells
 * (src/MixtureComp.cpp:494-573, src/OCPFluidMethod.cpp:1108-1187), including
 * the skip-stability decision CalFtypeFIM (src/AcceleratePVT.cpp:96-120) and
 * CalSkipForNextStep (src/MixtureComp.cpp:5234-5254) on `skip`.
 * form: one of OCPF_FORM_*. Asynchronous on `stream`. The plain form
 * allocates nothing; the batched forms use the context's scratch (see
 * ocpf_reserve). */
int ocpf_flash_fim(ocpf_ctx* ctx, int64_t ncell, const ocpf_fim_in* in, ocpf_skip* skip,
                   ocpf_fim_out* out, int form, void* stream);

/* Pre-allocates the context's device scratch (per-cell equilibrium buffer
 * and work queue, about 0.3 KB per cell) for batches of up to ncell cells,
 * so that later calls of the batched forms allocate nothing (e.g. before
 * capturing them in a CUDA graph). Without it the scratch grows on the
 * first call that needs more. No reference counterpart (the reference keeps
 * its scratch inside each MixtureComp object). */
int ocpf_reserve(ocpf_ctx* ctx, int64_t ncell);

/* The batched form (OCPF_FORM_BATCHED) for callers that cannot allocate
 * device memory: applications that own all of the GPU's memory through their
 * own pool or arena, run under a fixed device-memory budget, or must not let
 * a flash call synchronise the device (cudaMalloc and cudaFree may). Its
 * scratch -- per-cell phase state and cell lists, ~1.9 KB per cell for up to
 * 12 components -- lives in one array compiled into the library, of
 * OCPF_NOALLOC_MAX_CELLS cells (about 7.6 MB, held on every GPU that loads
 * the library until the process exits). The caller passes inputs and outputs
 * as for ocpf_flash_fim; the call allocates nothing and is asynchronous on
 * `stream`. Returns OCPF_ERANGE, without touching the GPU, when ncell exceeds
 * OCPF_NOALLOC_MAX_CELLS.
 * The first call on a device looks up the array's device address there
 * (cudaGetSymbolAddress), so make that first call before any stream capture.
 * That address is kept for the life of the process: after cudaDeviceReset
 * (or anything else that destroys the device's primary context) it is
 * stale, and the next call would write to memory that no longer belongs to
 * the library -- do not reset a device between calls of this function.
 * Every call on a device uses the same array and leaves its contents behind;
 * the call clears what must start empty itself. Calls whose work overlaps on
 * the GPU (two streams, or two host threads) race on the array and corrupt
 * each other: issue them one after another on one stream.
 * No counterpart in the reference (it keeps its scratch inside each
 * MixtureComp object on the host). */
int ocpf_flash_fim_noalloc(ocpf_ctx* ctx, int64_t ncell, const ocpf_fim_in* in, ocpf_skip* skip,
                           ocpf_fim_out* out, void* stream);

/* Batched MixtureComp::FlashIMPEC + IsoT_IMPEC::PassFlashValue over ncell
 * cells (src/MixtureComp.cpp:444-492, src/OCPFluidMethod.cpp:264-305): the
 * IMPEC flash type (skip or full; no two-phase warm type), the same phase
 * equilibrium as the FIM call, then the volume derivatives vfi / vfP and the
 * phase properties without dXsdXp or property partials. Forms and
 * asynchrony as ocpf_flash_fim. */
int ocpf_flash_impec(ocpf_ctx* ctx, int64_t ncell, const ocpf_impec_in* in, ocpf_skip* skip,
                     ocpf_impec_out* out, int form, void* stream);

/* Batched MixtureComp::InitFlashFIM + IsoT_FIM::PassFlashValue over ncell
 * cells (src/MixtureComp.cpp:261-353, src/OCPFluidMethod.cpp:1095-1106): a
 * full flash of z (strict stability, no skip test, no warm start), the
 * hydrocarbon moles Nh = Vpore (1 - S_w) / vf and the water moles
 * Vpore S_w xi_w that fill the pore volume, then FlashFIM's derivatives and
 * outputs. Ni [numCom][ncell] receives the moles (what IsoT_FIM::InitFlash
 * copies back into Bulk::Ni); it may alias in->zi, and out->S may alias
 * in->S. The skip cache is written as FlashFIM writes it. Forms and
 * asynchrony as ocpf_flash_fim. As in the reference, out->nj of a
 * hydrocarbon phase holds its mole fraction (CopyPhase runs before the
 * moles are scaled); the other outputs are per cell as after FlashFIM. */
int ocpf_init_flash_fim(ocpf_ctx* ctx, int64_t ncell, const ocpf_init_in* in, ocpf_skip* skip, double* Ni,
                        ocpf_fim_out* out, int form, void* stream);

/* Batched MixtureComp::InitFlashIMPEC + IsoT_IMPEC::PassFlashValue
 * (src/MixtureComp.cpp:195-259, src/OCPFluidMethod.cpp:251-262): as
 * ocpf_init_flash_fim with the IMPEC outputs of ocpf_flash_impec. */
int ocpf_init_flash_impec(ocpf_ctx* ctx, int64_t ncell, const ocpf_init_in* in, ocpf_skip* skip, double* Ni,
                          ocpf_impec_out* out, int form, void* stream);

/* The flash of a subset of the bulks: the calls of IsoT_AIMc::CalFlashI
 * (src/OCPFluidMethod.cpp:4293-4314, FlashFIM + PassFlashValue on the
 * implicit bulks) and CalFlashEa / CalFlashEp (:4257-4291, FlashIMPEC on
 * the explicit bulks). in / skip / out are the full arrays of ncell cells
 * (the layouts of ocpf_flash_fim / ocpf_flash_impec, stride ncell); idx
 * [nsub] (device, distinct, in [0, ncell); others are skipped) lists the
 * cells to flash. Only the listed cells are read and written; each gets
 * exactly what the full call gives it. The listed cells are gathered into
 * compact copies held by the context (about 2.4 KB per cell for 6
 * components, grown on demand; a growth synchronises the device), flashed
 * in the chosen form and scattered back. Asynchronous on `stream`. */
int ocpf_flash_fim_subset(ocpf_ctx* ctx, int64_t nsub, const int64_t* idx, int64_t ncell, const ocpf_fim_in* in,
                          ocpf_skip* skip, ocpf_fim_out* out, int form, void* stream);
int ocpf_flash_impec_subset(ocpf_ctx* ctx, int64_t nsub, const int64_t* idx, int64_t ncell,
                            const ocpf_impec_in* in, ocpf_skip* skip, ocpf_impec_out* out, int form, void* stream);

/* Batched MixtureComp::FlashFIMn + IsoT_FIMn::PassFlashValue over ncell
 * cells (src/MixtureComp.cpp:575-695, src/OCPFluidMethod.cpp:3152-3196),
 * the flash of the FIM formulation whose secondary variables are the
 * saturations and the phase moles n_ij: the same flash type and phase
 * equilibrium as ocpf_flash_fim, then (CaldXsdXpAPI03, :4495-4631)
 * out->dSec_dPri holds, per existing hydrocarbon phase in phase order, the
 * rows dS_j/d(P, N), then dS_w/d(P, N), then the rows dn_ij/d(P, N)
 * (bRowSizedSdP = NP + 1 + NP nc rows of numCom + 1 columns); xix, rhox and
 * mux are the derivatives per n_ij (CalXiPn_partial, CalRhoPn_partial,
 * CalMuPnLBC_partial), vfP and vfi follow CalVfiVfp_full03, and
 * pVnumCom[w] = 0. out->nj (required here) receives the phase moles.
 * res [3 (numCom + 1)][ncell] receives the first bRowSizedSdP entries of
 * the solve's residual column (Bulk::res_n; zeros for a single hydrocarbon
 * phase) and resPc [ncell] the reference's resPc (Bulk::resPc). The
 * reference reads its njin and phaseExistin arguments only to form a phase
 * count its branch never uses; they are not inputs here. The skip cache is
 * read and written as by ocpf_flash_fim. Forms and asynchrony as
 * ocpf_flash_fim. */
int ocpf_flash_fimn(ocpf_ctx* ctx, int64_t ncell, const ocpf_fim_in* in, ocpf_skip* skip,
                    ocpf_fim_out* out, double* res, double* resPc, int form, void* stream);

/* Batched MixtureComp::InitFlashFIMn + IsoT_FIMn::PassFlashValue
 * (src/MixtureComp.cpp:355-442, src/OCPFluidMethod.cpp:3129-3150): the
 * initialisation of ocpf_init_flash_fim with the outputs of
 * ocpf_flash_fimn. */
int ocpf_init_flash_fimn(ocpf_ctx* ctx, int64_t ncell, const ocpf_init_in* in, ocpf_skip* skip, double* Ni,
                         ocpf_fim_out* out, double* res, double* resPc, int form, void* stream);

/* Schedules of ocpf_flash_fim_regions for the batched forms. */
#define OCPF_SCHED_ONE_LAUNCH 0 /* one launch sequence over every region: each step is one kernel over all
                                   regions' cells, the persistent kernels' warps drain one region's work
                                   and move on to the next (at most 4 regions of 3, 6, 9 or 12 components;
                                   otherwise the streams schedule is used) */
#define OCPF_SCHED_STREAMS 1    /* one launch sequence per region, overlapped on the regions' own streams */

/* Launch shape of the batched forms of one context, and the schedule of the
 * ocpf_flash_fim_regions calls it leads (as ctx[0]). Every field changes
 * only which GPU thread handles which cell, except slow_threads, which
 * runs the split restarts of the few cells that need them on one thread per
 * cell instead of one warp per cell (the two paths agree to rounding). No
 * reference counterpart. */
typedef struct {
    int32_t block;        /* threads per block of the thread-per-item kernels: 64 or 128 (default 128) */
    int32_t persist_pct;  /* resident blocks per SM of the persistent kernels, in percent of what their
                             registers allow: 1..100 (default 100) */
    int32_t slow_threads; /* split restarts: 0 one warp per cell (default), 1 one thread per cell */
    int32_t schedule;     /* OCPF_SCHED_* (default OCPF_SCHED_ONE_LAUNCH) */
    float   ms;           /* ocpf_autotune: the chosen configuration's time per call; 0 when set by hand */
    int32_t pad;
} ocpf_tuning;

int ocpf_get_tuning(const ocpf_ctx* ctx, ocpf_tuning* t);
int ocpf_set_tuning(ocpf_ctx* ctx, const ocpf_tuning* t);

/* Autotuner: times the batched launch of `form` (OCPF_FORM_BATCHED, _MIXED or
 * _FAST) over these nreg regions (nreg = 1: one context's ocpf_flash_fim)
 * for every candidate launch shape -- block 64 / 128, persistent grids at
 * 50 / 100 % of their resident limit, split restarts on one warp / one
 * thread per cell and, for several regions, both schedules -- and keeps the
 * fastest in every context (*best receives it). The runs read the caller's
 * inputs and skip cache but write only the tuner's own copies: nothing of
 * the caller's arrays changes. It allocates those copies (about 2.3 KB per
 * cell for 6 components) for its duration and synchronises `stream`.
 * `reps` timed runs per candidate (after one untimed), at least 1. */
int ocpf_autotune(int nreg, ocpf_ctx* const* ctx, const int64_t* ncell, const ocpf_fim_in* in, const ocpf_skip* skip,
                  int form, int reps, void* stream, ocpf_tuning* best);

/* Several PVT regions at once -- the batched counterpart of a Bulk whose
 * cells belong to different regions (flashCal[PVTNUM[n]] in
 * src/OCPFluidMethod.cpp:1108-1120), with the cells grouped by region.
 * Region r flashes ncell[r] cells of in[r] / skip[r] / out[r] through
 * ctx[r] (distinct contexts; fluids of different component counts may be
 * mixed). The batched forms run as one launch sequence over all regions
 * (OCPF_SCHED_ONE_LAUNCH, the default, replayed from a CUDA graph while the
 * arguments stay the same) or as one sequence per region on the regions'
 * own streams (OCPF_SCHED_STREAMS), as ctx[0]'s tuning says; the plain form
 * always takes the streams. The call is asynchronous on `stream` like
 * ocpf_flash_fim. skip may be null when no region uses the skip cache.
 * With the streams schedule the results equal one ocpf_flash_fim per region
 * bit for bit; the one-launch kernels evaluate the same expressions but are
 * compiled apart (the compiler fuses multiply-adds per kernel), so they
 * agree to rounding. */
int ocpf_flash_fim_regions(int nreg, ocpf_ctx* const* ctx, const int64_t* ncell, const ocpf_fim_in* in,
                           ocpf_skip* skip, ocpf_fim_out* out, int form, void* stream);

/* Same call with every array in HOST memory (pinned memory is faster). The
 * cells are streamed through device staging buffers owned by the context in
 * chunks of 131,072 cells, copies overlapping the flash on four streams.
 * Each chunk goes to the first stream whose previous chunk is back, so a
 * chunk with a long restart chain holds back no other. The call returns
 * after the results are back in host memory. The staging buffers are allocated on the
 * first call (and grown if a larger chunk is requested) and kept until
 * ocpf_destroy. */
int ocpf_flash_fim_host(ocpf_ctx* ctx, int64_t ncell, const ocpf_fim_in* in, ocpf_skip* skip,
                        ocpf_fim_out* out, int form);

/* ---- Last-time-step copies -------------------------------------------
 * IsoT_FIM::UpdateLastTimeStep (src/OCPFluidMethod.cpp:2915-2960) keeps a
 * copy of every Bulk array the flash writes, and ResetToLastTimeStep
 * (:2859-2897) puts it back when a time step is cut; SkipStaAnaly does the
 * same for its cache (src/AcceleratePVT.cpp:122-138). Here `last` and
 * `last_skip` are the caller's arrays in the layouts of ocpf_fim_out and
 * ocpf_skip for the same ncell and nc (hydrocarbon components):
 *   ocpf_update_last_step:   last <- cur, last_skip <- skip;
 *   ocpf_reset_to_last_step: cur <- last, skip <- last_skip.
 * Every field set in both structs is copied, the optional diagnostics
 * included, dSec_dPri whole ([3*(numCom+1)^2][ncell]); a field set in only
 * one of the two is OCPF_EINVAL, as are skip and last_skip not both set or
 * both null and a source overlapping its destination. One kernel launch
 * copies all the arrays, asynchronously on `stream`. The Bulk arrays
 * outside the flash (P, Ni, Pj, Pc, kr and the rock's) are the caller's:
 * ocpf_copy_arrays copies any of them in one launch as well. */
#define OCPF_COPY_MAX 64 /* array pairs of one copy launch */
int ocpf_update_last_step(int nc, int64_t ncell, const ocpf_fim_out* cur, const ocpf_skip* skip,
                          const ocpf_fim_out* last, const ocpf_skip* last_skip, void* stream);
int ocpf_reset_to_last_step(int nc, int64_t ncell, const ocpf_fim_out* cur, const ocpf_skip* skip,
                            const ocpf_fim_out* last, const ocpf_skip* last_skip, void* stream);

/* Copies narr (at most OCPF_COPY_MAX) device arrays, src[i] to dst[i] of
 * bytes[i] bytes, in one kernel launch on `stream`. Arrays of 0 bytes and
 * pairs with dst[i] == src[i] are skipped; a null pointer of a non-empty
 * pair, a negative size or a source overlapping its destination is
 * OCPF_EINVAL (and nothing is launched). */
int ocpf_copy_arrays(int narr, void* const* dst, const void* const* src, const int64_t* bytes, void* stream);

/* Device time (ms) of the last ocpf_flash_fim's flash kernel, measured with
 * CUDA events on its stream; waits for that kernel to finish. */
int ocpf_last_kernel_ms(ocpf_ctx* ctx, float* ms);

/* With on != 0, every later ocpf_flash_fim of a batched form records the
 * events ocpf_last_phase_ms reads, and launches its kernel sequence directly
 * instead of replaying it from the context's CUDA graph (events recorded by
 * a replayed graph cannot be timed against each other). Off by default. No
 * reference counterpart (measurement utility). */
int ocpf_set_part_timing(ocpf_ctx* ctx, int on);

/* The parts of the last ocpf_flash_fim in a batched form with part timing
 * on (device time, ms, CUDA events on its stream; waits for the call to
 * finish; zeros otherwise): ms[0] the
 * sequence up to the split-restart path (set-up, stability tests, the
 * split's first try), ms[1] the restart path (the few cells whose split
 * restarts), ms[2] finalize (properties, derivatives, copy-out). No
 * reference counterpart (measurement utility). */
int ocpf_last_phase_ms(ocpf_ctx* ctx, float* ms);

/* Number of kernels the last flash call on this context launched (1 for
 * the plain form; for the batched forms the kernel nodes of the replayed
 * launch sequence), or -1 when unknown (the first call of a sequence, which
 * launches directly, or a call inside the caller's own stream capture). A
 * measurement aid; no reference counterpart. */
int ocpf_last_launch_count(ocpf_ctx* ctx, int* n);

/* Measures the device's FMA throughput (TFLOP/s, FMA = 2 flops) in FP64
 * (bits = 64) or FP32 (bits = 32) with a short register-only kernel: the
 * compute-roofline denominator for the flash kernels. No reference
 * counterpart (measurement utility). */
int ocpf_measure_fma_peak(int device, int bits, double* tflops);

/* ---- Learned initialiser (no counterpart in the reference) -------------
 * A small MLP predicts, from a cell's (ln P, T, z), whether its feed is
 * unstable (a logit) and the ln K of the split. Layers nin -> 64 -> 64 ->
 * nout with SiLU, BF16 weights and activations, FP32 accumulation, run on the
 * tensor cores. For an NC-component fluid nin = NC + 2 and nout = NC + 1
 * (output 0: logit of "unstable"; outputs 1..NC: ln K_i = ln(y_i / x_i),
 * vapour over liquid). Parameters are one FP32 vector of
 * ocpf_mlp_param_count() floats: W1[64][16] b1[64] W2[64][64] b2[64]
 * W3[16][64] b3[16], row-major [out][in], zero beyond nin / nout.
 * Arrays are device memory, feature-major: x[f * n + s]. */
#define OCPF_MLP_HIDDEN 64
#define OCPF_MLP_MAX_IO 16

int ocpf_mlp_param_count(void);

/* y[j * n + s] = MLP(x[:, s])_j for j < nout. */
int ocpf_mlp_forward(int nin, int nout, int64_t n, const float* params, const float* x, float* y, void* stream);

/* Adds to grad (ocpf_mlp_param_count() floats) the gradient of the mean loss
 *   1/n sum_s [ softplus(o_0) - t_0 o_0 + lnk_weight w_s / (nout-1) sum_{j>=1} (o_j - t_j)^2 ]
 * (targets t[j * n + s], t_0 in {0, 1}; w_s = wmask[s], 0 for samples with
 * no split) and adds the two loss sums (logistic, ln K) to loss[0], loss[1]. */
int ocpf_mlp_grad(int nin, int nout, int64_t n, const float* params, const float* x, const float* target,
                  const float* wmask, float lnk_weight, float* grad, float* loss, void* stream);

/* One Adam step (beta 0.9 / 0.999, eps 1e-8, bias-corrected at `step` >= 1)
 * of the FP32 parameters from grad, with moment buffers m, v; zeroes grad. */
int ocpf_mlp_adam(float* params, float* grad, float* m, float* v, int step, float lr, void* stream);

/* Attaches a trained initialiser to a context for OCPF_FORM_FAST: params
 * (host, ocpf_mlp_param_count() floats), the input normalisation
 * (feature f = (raw_f - in_mean[f]) / in_scale[f] for the raw features
 * ln(P / psia), T / degF, z_1..z_NC; host arrays of NC + 2) and the
 * confidence at or above which a fresh cell's predicted instability is
 * acted on (the split starts from the predicted K; the stability test runs
 * only if that split fails). Without one, OCPF_FORM_FAST runs as
 * OCPF_FORM_MIXED. */
int ocpf_set_initializer(ocpf_ctx* ctx, const float* params, const float* in_mean, const float* in_scale,
                         float confidence);

/* Measures, on one thread with clock64, the latency in cycles of FP64
 * operations that bound a single cell's chain of dependent iterations:
 * cycles[0] division, [1] division when twelve independent ones are issued
 * together (per division), [2] FMA, [3] exp, [4] log, [5] acos + cos. No
 * reference counterpart (measurement utility). */
int ocpf_measure_fp64_latency(int device, double* cycles);

/* ---------------------------------------------------------------------
 * Relative permeability and capillary pressure after the flash
 * (IsoT_FIM::CalKrPc / IsoT_IMPEC::CalKrPc, src/OCPFluidMethod.cpp:
 * 1189-1199 and :311-319, with the compositional model's default flow unit
 * FlowUnit_ODGW01, src/FlowUnit.cpp:183-349, chosen by Bulk::Setup when
 * there is no SOF3 table and no miscibility, src/Bulk.cpp:271-279).
 * --------------------------------------------------------------------- */

/* The SWOF and SGOF tables of one saturation region, in host memory, rows
 * as the keywords list them (4 columns, row-major): Sw, krw, krow, Pcow and
 * Sg, krg, krog, Pcgo. The first column of each must not decrease. */
typedef struct {
    int32_t       nrow_swof, nrow_sgof;
    const double* swof;
    const double* sgof;
} ocpf_satfunc;

/* The SWFN, SGFN and SOF3 tables of one saturation region (3 columns,
 * row-major, as the keywords list them): Sw, krw, Pcow; Sg, krg, Pcgo;
 * So, krow, krog. The reference uses this family (FlowUnit_ODGW02) as soon
 * as SOF3 is given (src/Bulk.cpp:271-279). */
typedef struct {
    int32_t       nrow_swfn, nrow_sgfn, nrow_sof3, pad;
    const double* swfn;
    const double* sgfn;
    const double* sof3;
} ocpf_satfunc3;

typedef struct ocpf_krpc ocpf_krpc;

/* Device inputs: P [ncell], the flash's S [3][ncell] (oil, gas, water), and
 * the region of each cell (Bulk::SATNUM) or null for region 0. */
typedef struct {
    const double*  P;
    const double*  S;
    const int32_t* satnum;
} ocpf_krpc_in;

/* Device outputs (Bulk::kr, Pc, Pj, dKr_dS, dPcj_dS): kr, Pc, Pj
 * [3][ncell]; dKr_dS, dPcj_dS [9][ncell] with entry 3 j + k = d/dS_k of
 * phase j. Both derivative arrays null: the IMPEC call (no derivatives). */
typedef struct {
    double* kr;
    double* Pc;
    double* Pj;
    double* dKr_dS;
    double* dPcj_dS;
} ocpf_krpc_out;

/* Builds the device tables of nregion regions (FlowUnit_ODGW01's
 * constructor, src/FlowUnit.cpp:183-203): OCPF_EINVAL for a table with
 * fewer than 2 rows or a decreasing first column, OCPF_EUNSUPPORTED when
 * the tables exceed 48 KB together. */
int ocpf_krpc_create(const ocpf_satfunc* regions, int nregion, int device, ocpf_krpc** out);

/* The same for FlowUnit_ODGW02 (src/FlowUnit.cpp:522-535): ocpf_cal_krpc on
 * the handle then evaluates SWFN at S_w, SGFN at S_g and SOF3 at S_o, with
 * the reference's two oil models kept as they are: with derivative outputs
 * (CalKrPcDeriv, :569-652) Stone II from kroMax = SOF3's last krow, whose
 * derivative enters dKr_dS[0] (d kro / d S_o) alone; without (CalKrPc,
 * :537-567) the default model (Sg krog + (Sw - Swco) krow) / (Sg + Sw - Swco),
 * kroMax where that denominator is at most 1e-8. Same error codes. */
int ocpf_krpc_create_sof3(const ocpf_satfunc3* regions, int nregion, int device, ocpf_krpc** out);
int ocpf_krpc_destroy(ocpf_krpc* k);

/* For every cell: SWOF at S_w and SGOF at S_g (OCPTable::Eval_All, linear
 * interpolation, flat outside the table), Stone II kro (negative values
 * clipped to 0 with their derivatives), Pc = (0, Pcgo, -Pcow), Pj = P + Pc,
 * and with derivative outputs CalKrPcDeriv's dKr_dS and dPcj_dS. A cell
 * whose region does not exist gets NaN outputs. Results equal the
 * reference's bit for bit. Asynchronous on `stream`. */
int ocpf_cal_krpc(ocpf_krpc* k, int64_t ncell, const ocpf_krpc_in* in, const ocpf_krpc_out* out, void* stream);

/* ---------------------------------------------------------------------
 * The consumer of the flash's derivatives: the bulk part of the FIM
 * Jacobian (IsoT_FIM::AssembleMatBulksNew, src/OCPFluidMethod.cpp:
 * 1569-1840) and the upstream choice that precedes it (src/BulkConn.cpp:
 * 170-215).
 * --------------------------------------------------------------------- */

typedef struct ocpf_conn ocpf_conn;

/* The Bulk arrays the assembly reads, on the device, in the flash's
 * layouts ([field][nbulk]): the flash outputs, CalKrPc's (kr, Pj [3];
 * dKr_dS, dPcj_dS [9]), and the rock: bulk volume v, dporosity/dP poroP and
 * depth [nbulk]. S and rho are read by ocpf_fim_upwind only. */
typedef struct {
    const uint32_t* phaseExist; /* [3] */
    const uint32_t* pSderExist; /* [3] */
    const uint32_t* pVnumCom;   /* [3] */
    const double*   S;          /* [3] */
    const double*   rho;        /* [3] */
    const double*   xi;         /* [3] */
    const double*   mu;         /* [3] */
    const double*   muP;        /* [3] */
    const double*   xiP;        /* [3] */
    const double*   rhoP;       /* [3] */
    const double*   xij;        /* [3*numCom] */
    const double*   rhox;       /* [3*numCom] */
    const double*   xix;        /* [3*numCom] */
    const double*   mux;        /* [3*numCom] */
    const double*   dSec_dPri;  /* [3*(numCom+1)^2], bRowSizedSdP rows used */
    const double*   vfP;        /* [1] */
    const double*   vfi;        /* [numCom] */
    const double*   kr;         /* [3] */
    const double*   Pj;         /* [3] */
    const double*   dKr_dS;     /* [9] */
    const double*   dPcj_dS;    /* [9] */
    const double*   v;          /* [1] */
    const double*   poroP;      /* [1] */
    const double*   depth;      /* [1] */
} ocpf_jac_bulk;

/* Device outputs, blocks of (numCom+1) x (numCom+1) entries, entry
 * r*(numCom+1)+c as the field index: diag [(numCom+1)^2][nbulk] (the
 * accumulation block plus, in connection order, each incident connection's
 * contribution, as the reference's AddDiag calls sum them); offEB and offBE
 * [(numCom+1)^2][nconn]: the blocks at (row eId, column bId) and (row bId,
 * column eId) of each connection (LinearSystem::NewOffDiag's). */
typedef struct {
    double* diag;
    double* offEB;
    double* offBE;
} ocpf_jac_out;

/* The connections of a grid (BulkConn: begin and end bulk and area of each,
 * host arrays), copied to `device` with the per-bulk list of incident
 * connections the diagonal blocks are gathered through. OCPF_EINVAL for a
 * bulk index outside [0, nbulk) or a connection from a bulk to itself. */
int ocpf_conn_create(int64_t nbulk, int64_t nconn, const int64_t* bId, const int64_t* eId, const double* area,
                     int device, ocpf_conn** out);
int ocpf_conn_destroy(ocpf_conn* conn);

/* Upstream bulk (upblock [3][nconn]) and mean density (upblock_rho
 * [3][nconn]) of every connection and phase from S, rho, Pj, phaseExist and
 * depth (BulkConn's upwind choice, src/BulkConn.cpp:170-215). Results equal
 * the reference's bit for bit. Asynchronous on `stream`. */
int ocpf_fim_upwind(ocpf_conn* conn, const ocpf_jac_bulk* bulk, int32_t* upblock, double* upblock_rho, void* stream);

/* The bulk part of the FIM Jacobian for time step dt (nc hydrocarbon
 * components: 3, 6, 9 or 12): per connection the flux derivatives of both
 * ends, dt (dF/dXp + dF/dXs dSec_dPri), and per bulk the accumulation plus
 * the diagonal contributions. Each operation is rounded as written in the
 * reference, in its order; the dense product sums in order (the reference's
 * BLAS dgemm may round its sums differently). Connections with shapes no
 * flash writes get NaN blocks. Asynchronous on `stream`. */
int ocpf_fim_jacobian(ocpf_conn* conn, int nc, double dt, const ocpf_jac_bulk* bulk, const int32_t* upblock,
                      const double* upblock_rho, ocpf_jac_out* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OCP_FLASH_H */
