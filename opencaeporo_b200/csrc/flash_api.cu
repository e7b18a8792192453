// flash_api.cu -- the C ABI of include/ocp_flash.h: context set-up (the
// derived per-fluid constants of MixtureComp's constructor), the batched
// FlashFIM launch on device buffers, and the pipelined host-buffer variant.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <chrono>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "flash_multi.cuh"

namespace ocpf {

// Per-NC launchers, one translation unit each (flash_plain_ncN.cu).
#define OCPF_DECL_PLAIN(N)                                                                        \
    cudaError_t launch_plain_nc##N(const FluidConst& F, int64_t count, int64_t stride,            \
                                   const ocpf_fim_in& in, const ocpf_skip& sk,                     \
                                   const ocpf_fim_out& out, const FlashTail& tail, unsigned blocks, \
                                   int bs, cudaStream_t st);
OCPF_DECL_PLAIN(3)
OCPF_DECL_PLAIN(6)
OCPF_DECL_PLAIN(9)
OCPF_DECL_PLAIN(12)

using PlainLauncher = cudaError_t (*)(const FluidConst&, int64_t, int64_t, const ocpf_fim_in&,
                                      const ocpf_skip&, const ocpf_fim_out&, const FlashTail&, unsigned, int,
                                      cudaStream_t);

// Batched-form launch sequences (flash_phased_ncN.cu).
#define OCPF_DECL_PHASED(N)                                                                                 \
    cudaError_t launch_phased_nc##N(const FluidConst& F, const PhasedArgs& a, const LaunchTune& t, cudaStream_t st, \
                                    const cudaEvent_t* marks, const SideStreams* side);                              \
    int         phased_state_doubles_nc##N();
OCPF_DECL_PHASED(3)
OCPF_DECL_PHASED(6)
OCPF_DECL_PHASED(9)
OCPF_DECL_PHASED(12)

using PhasedLauncher = cudaError_t (*)(const FluidConst&, const PhasedArgs&, const LaunchTune&, cudaStream_t,
                                       const cudaEvent_t*, const SideStreams*);

static PhasedLauncher phased_kernel(int nc, int* ndbl)
{
    switch (nc) {
        case 3: *ndbl = phased_state_doubles_nc3(); return launch_phased_nc3;
        case 6: *ndbl = phased_state_doubles_nc6(); return launch_phased_nc6;
        case 9: *ndbl = phased_state_doubles_nc9(); return launch_phased_nc9;
        case 12: *ndbl = phased_state_doubles_nc12(); return launch_phased_nc12;
        default: return nullptr;
    }
}

static PlainLauncher plain_kernel(int nc)
{
    switch (nc) {
        case 3: return launch_plain_nc3;
        case 6: return launch_plain_nc6;
        case 9: return launch_plain_nc9;
        case 12: return launch_plain_nc12;
        default: return nullptr;
    }
}

// ------------------------------------------------------- constant block

bool make_fluid_const(const ocpf_fluid& in, FluidConst& f)
{
    const int nc = in.nc;
    if (nc < 2 || nc > MAXNC) return false;
    std::memset(&f, 0, sizeof(f));
    f.nc           = nc;
    f.use_skip     = in.use_skip ? 1 : 0;
    f.rr_maxit     = in.rr_maxit;
    f.ssmsta_maxit = in.ssmsta_maxit;
    f.nrsta_maxit  = in.nrsta_maxit;
    f.ssmsp_maxit  = in.ssmsp_maxit;
    f.nrsp_maxit   = in.nrsp_maxit;
    f.rr_tol       = in.rr_tol;
    f.ssmsta_tol2  = in.ssmsta_tol * in.ssmsta_tol;  // src/MixtureComp.cpp:143
    f.ssmsta_eyt   = in.ssmsta_eyt;
    f.nrsta_tol    = in.nrsta_tol;
    f.ssmsp_tol2   = in.ssmsp_tol * in.ssmsp_tol;
    f.nrsp_tol     = in.nrsp_tol;
    if (in.rr_maxit < 0 || in.ssmsta_maxit < 0 || in.nrsta_maxit < 0 || in.ssmsp_maxit < 0 ||
        in.nrsp_maxit < 0)
        return false;
    for (int i = 0; i < nc; i++) {
        if (!(in.Tc[i] > 0) || !(in.Pc[i] > 0) || !(in.Vc[i] > 0) || !(in.MW[i] > 0)) return false;
        f.Tc[i]     = in.Tc[i];
        f.Pc[i]     = in.Pc[i];
        f.Vc[i]     = in.Vc[i];
        f.Vcvis[i]  = in.Vc[i];  // no VCRITVIS/ZCRITVIS: Vcvis = Vc (src/MixtureComp.cpp:98-106)
        f.MW[i]     = in.MW[i];
        f.Acf[i]    = in.Acf[i];
        f.OmegaA[i] = in.OmegaA[i];
        f.OmegaB[i] = in.OmegaB[i];
        // VSHIFT scaling, src/MixtureComp.cpp:89-93
        f.Vshift[i] = in.Vshift[i] * (GAS_CONSTANT * in.OmegaB[i] * in.Tc[i] / in.Pc[i]);
        // PR m(omega), src/MixtureComp.cpp:923-929
        const double acf = in.Acf[i];
        f.mwi[i] = (acf <= 0.49) ? 0.37464 + 1.54226 * acf - 0.26992 * std::pow(acf, 2)
                                 : 0.379642 + 1.48503 * acf - 0.164423 * std::pow(acf, 2) +
                                       0.016667 * std::pow(acf, 3);
        f.sqrtMW[i]  = std::sqrt(in.MW[i]);
        f.muAux1I[i] = 5.4402 * std::pow(in.Tc[i], 1.0 / 6) / std::pow(in.Pc[i], 2.0 / 3);
        f.lbc1[i]    = 5.4402 * std::pow(in.Tc[i], 1.0 / 6);
        f.lbc2[i]    = std::pow(in.Pc[i], 2.0 / 3);
        for (int k = 0; k < nc; k++) {
            if (in.BIC[i * nc + k] != in.BIC[k * nc + i]) return false;
            f.omb[i * MAXNC + k]  = 1 - in.BIC[i * nc + k];
            f.ombf[i * MAXNC + k] = (float)f.omb[i * MAXNC + k];
        }
    }
    for (int k = 0; k < 5; k++) {
        f.L[k]    = in.LBCcoef[k] * 10;  // src/MixtureComp.cpp:108-111
        f.pvtw[k] = in.pvtw[k];
    }
    f.std_rho_w = in.std_rho_w;
    return true;
}

}  // namespace ocpf

using namespace ocpf;

// Parts of the host-buffer path in flight at once, each with its own
// stream, staging buffers and scratch: a chunk that holds a long restart
// chain then delays only the chunks of its own part.
constexpr int HOST_PARTS = 4;

struct ocpf_ctx {
    int         device;
    FluidConst  fc;
    cudaEvent_t ev0, ev1;
    // the batched sequence's parts in the last timed call: marks[0] before
    // and marks[1] after its split-restart kernel
    cudaEvent_t marks[2];
    bool        marked;
    bool        part_timing;  // ocpf_set_part_timing: record the marks (launches directly)
    bool        timed;
    // host-path staging (device) buffers, grown on demand
    int64_t     stage_cap;
    void*       stage;
    cudaStream_t hs[HOST_PARTS];
    cudaEvent_t  hdone[HOST_PARTS];  // recorded after each part's last copy-out
    // batched-form scratch: per-cell phase state, cell lists and list
    // counters, in parts of part_cap cells (the host path uses HOST_PARTS parts)
    int64_t     eq_cap;    // total cells the scratch holds
    void*       eq;
    // learned initialiser parameters (device, MLP_NPARAM floats) or null
    float*      mlp;
    // ocpf_flash_fim_regions: this region's stream and its fork/join events
    cudaStream_t rs;
    cudaEvent_t  evf, evj;
    // the batched forms' launch sequence as a CUDA graph, replayed while the
    // call's arguments stay the same (captured on a private stream)
    int64_t         launches;  // batched-form calls so far
    cudaStream_t    gs;
    cudaGraphExec_t gexec;
    PhasedArgs      gkey;
    LaunchTune      gtune;
    bool            gmark;   // the captured sequence records the part marks
    bool            gvalid;
    // launch shape of the batched forms (ocpf_set_tuning / ocpf_autotune)
    // and, for ocpf_flash_fim_regions led by this context, the schedule
    LaunchTune tune;
    int32_t    sched;
    float      tune_ms;
    // ocpf_flash_fim_regions' one-launch sequence as a CUDA graph, keyed by
    // its arguments (held by the first region's context)
    cudaGraphExec_t mgexec;
    MultiArgs*      mgkey;
    LaunchTune      mgtune;
    int32_t         mgkernels;
    int32_t         gkernels;      // kernel nodes of the captured graph
    int32_t         last_kernels;  // kernels the last call launched, -1 unknown
    // subset calls: compact device copies of the listed cells, grown on demand
    int64_t sub_cap;
    void*   sub;
    // the PH_EARLY schedule's side streams and fork/join events, created on
    // the first batched call
    SideStreams side;
    bool        side_ok;
};

static const char* kVersion = "opencaeporo-b200 flash 0.1 (sm_100a)";

extern "C" const char* ocpf_version(void) { return kVersion; }

extern "C" const char* ocpf_status_string(int code)
{
    switch (code) {
        case OCPF_OK: return "ok";
        case OCPF_EINVAL: return "invalid argument";
        case OCPF_ECUDA: return "CUDA runtime error";
        case OCPF_ENOMEM: return "device allocation failed";
        case OCPF_EUNSUPPORTED: return "unsupported";
        case OCPF_ERANGE: return "batch larger than OCPF_NOALLOC_MAX_CELLS";
        default: return "unknown";
    }
}

extern "C" int ocpf_create(const ocpf_fluid* fluid, int device, ocpf_ctx** ctx)
{
    if (!fluid || !ctx) return OCPF_EINVAL;
    *ctx = nullptr;
    FluidConst fc;
    if (!make_fluid_const(*fluid, fc)) return OCPF_EINVAL;
    if (!plain_kernel(fc.nc)) return OCPF_EUNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return OCPF_ECUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return OCPF_ECUDA;
    if (prop.major != 10) return OCPF_EUNSUPPORTED;  // built for sm_100a only
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return OCPF_ECUDA;
    ocpf_ctx* c = new (std::nothrow) ocpf_ctx();
    if (!c) return OCPF_ENOMEM;
    c->device    = device;
    c->fc        = fc;
    c->timed     = false;
    c->stage_cap = 0;
    c->stage     = nullptr;
    c->sub_cap   = 0;
    c->sub       = nullptr;
    for (auto& s : c->hs) s = nullptr;
    c->eq_cap    = 0;
    c->eq        = nullptr;
    c->mlp       = nullptr;
    c->rs        = nullptr;
    c->evf = c->evj = nullptr;
    c->launches  = 0;
    c->gkernels     = 0;
    c->last_kernels = -1;
    c->gs        = nullptr;
    c->gexec     = nullptr;
    c->gvalid    = false;
    c->gtune     = kDefaultTune;
    c->gmark     = false;
    c->tune      = kDefaultTune;
    c->sched     = OCPF_SCHED_ONE_LAUNCH;
    c->tune_ms   = 0;
    c->mgexec    = nullptr;
    c->mgkey     = nullptr;
    c->mgtune    = kDefaultTune;
    c->mgkernels = 0;
    c->marked      = false;
    c->part_timing = false;
    if (cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreate(&c->marks[0]) != cudaSuccess || cudaEventCreate(&c->marks[1]) != cudaSuccess) {
        delete c;
        cudaSetDevice(prev);
        return OCPF_ECUDA;
    }
    cudaSetDevice(prev);
    *ctx = c;
    return OCPF_OK;
}

extern "C" int ocpf_destroy(ocpf_ctx* c)
{
    if (!c) return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    cudaEventDestroy(c->ev0);
    cudaEventDestroy(c->ev1);
    cudaEventDestroy(c->marks[0]);
    cudaEventDestroy(c->marks[1]);
    if (c->stage) cudaFree(c->stage);
    if (c->sub) cudaFree(c->sub);
    if (c->eq) cudaFree(c->eq);
    if (c->mlp) cudaFree(c->mlp);
    if (c->rs) cudaStreamDestroy(c->rs);
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->mgexec) cudaGraphExecDestroy(c->mgexec);
    delete c->mgkey;
    if (c->gs) cudaStreamDestroy(c->gs);
    if (c->evf) cudaEventDestroy(c->evf);
    if (c->evj) cudaEventDestroy(c->evj);
    for (auto& s : c->hs)
        if (s) cudaStreamDestroy(s);
    for (auto& ev : c->hdone)
        if (ev) cudaEventDestroy(ev);
    for (int k = 0; k < 4; k++) {
        if (c->side.s[k]) cudaStreamDestroy(c->side.s[k]);
        if (c->side.fork[k]) cudaEventDestroy(c->side.fork[k]);
        if (c->side.join[k]) cudaEventDestroy(c->side.join[k]);
    }
    cudaSetDevice(prev);
    delete c;
    return OCPF_OK;
}

// The outputs every FIM-tail entry point writes (IsoT_FIM::PassFlashValue's).
static bool fim_out_ok(const ocpf_fim_out* o)
{
    return o && o->phaseNum && o->phaseExist && o->S && o->Nt && o->vf && o->vfP && o->vfi && o->rho && o->xi &&
           o->mu && o->rhoP && o->xiP && o->muP && o->xij && o->rhox && o->xix && o->mux && o->dSec_dPri &&
           o->bRowSizedSdP && o->pSderExist && o->pVnumCom;
}

// The outputs every IMPEC-tail entry point writes (IsoT_IMPEC::PassFlashValue's).
static bool impec_out_ok(const ocpf_impec_out* o)
{
    return o && o->phaseNum && o->phaseExist && o->S && o->Nt && o->vf && o->vfP && o->vfi && o->vj && o->rho &&
           o->xi && o->mu && o->xij;
}

static bool skip_ok(const ocpf_ctx* c, const ocpf_skip* sk)
{
    return !c->fc.use_skip || (sk && sk->flag && sk->minEig && sk->P && sk->T && sk->z);
}

// The IMPEC outputs as the FIM output record the kernels write through.
static ocpf_fim_out impec_as_fim(const ocpf_impec_out& o)
{
    ocpf_fim_out fo{};
    fo.phaseNum   = o.phaseNum;
    fo.phaseExist = o.phaseExist;
    fo.S          = o.S;
    fo.Nt         = o.Nt;
    fo.vf         = o.vf;
    fo.vfP        = o.vfP;
    fo.vfi        = o.vfi;
    fo.rho        = o.rho;
    fo.xi         = o.xi;
    fo.mu         = o.mu;
    fo.xij        = o.xij;
    fo.ePEC       = o.ePEC;
    fo.ftype      = o.ftype;
    fo.iters      = o.iters;
    fo.status     = o.status;
    return fo;
}

static bool fim_args_ok(const ocpf_ctx* c, const ocpf_fim_in* in, const ocpf_skip* sk,
                        const ocpf_fim_out* o)
{
    if (!in || !in->P || !in->T || !in->Ni || !in->S || !in->lastNP || !in->xij) return false;
    return fim_out_ok(o) && skip_ok(c, sk);
}

static size_t scratch_bytes_per_cell(int nc)
{
    int nd = 0;
    phased_kernel(nc, &nd);
    return state_bytes_per_cell(nd) + 4 * (size_t)L_COUNT;
}

static size_t part_bytes(int nc, int64_t cap)
{
    return ((scratch_bytes_per_cell(nc) * (size_t)cap + 2 * 4 * L_COUNT + 255) / 256 + 1) * 256;
}

// Grows the scratch to hold `parts` parts of `cap` cells each.
static int ensure_scratch(ocpf_ctx* c, int64_t cap, int parts = 1)
{
    const int64_t need = cap * parts;
    if (c->eq_cap >= need && c->eq) return OCPF_OK;
    if (c->eq) {
        cudaDeviceSynchronize();  // the old scratch may still be in use by queued work
        cudaFree(c->eq);
    }
    c->eq     = nullptr;
    c->eq_cap = 0;
    if (cudaMalloc(&c->eq, part_bytes(c->fc.nc, need) + 4096) != cudaSuccess) return OCPF_ENOMEM;
    c->eq_cap = need;
    return OCPF_OK;
}

// Part `part` of the scratch laid out for `cap` cells.
static void scratch_view(const ocpf_ctx* c, int part, int64_t cap, StateBuf& S, Lists& L)
{
    int nd = 0;
    phased_kernel(c->fc.nc, &nd);
    char* base = (char*)c->eq + (size_t)part * part_bytes(c->fc.nc, cap);
    S.cap      = cap;
    S.d        = (double*)base;
    S.i        = (int32_t*)(S.d + (size_t)nd * cap);
    L.cap      = cap;
    L.items    = S.i + (size_t)IF_COUNT * cap;
    L.ctr      = (uint32_t*)(L.items + (size_t)L_COUNT * cap);
}

// The batched forms launch ~40-60 kernels per call. From the second call of
// a context on (the first one also sets up each kernel's launch shape), the
// sequence is captured once into a CUDA graph on the context's private
// stream and replayed with one cudaGraphLaunch on the caller's stream while
// the arguments (sizes, device pointers, form) stay the same; a change
// re-captures (cudaGraphExecUpdate keeps the executable when only parameters
// differ). Work already captured by the caller's own stream capture, and the
// host path's alternating parts, launch directly.
// The side streams of the PH_EARLY schedule, created once per context.
static bool ensure_side(ocpf_ctx* c)
{
    if (c->side_ok) return true;
    // The side streams of trials 1-3 carry few cells, among them the ones
    // whose stability was hardest to decide and whose restart chains are
    // the call's critical path: their blocks are dispatched ahead of the
    // rest. (Stream 0 is not used: trial 0's cells split on the call's
    // stream.)
    int lo = 0, hi = 0;
    if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) lo = hi = 0;
    for (int k = 0; k < 4; k++) {
        if (!c->side.s[k] &&
            cudaStreamCreateWithPriority(&c->side.s[k], cudaStreamNonBlocking, k == 0 ? lo : hi) != cudaSuccess)
            return false;
        if (!c->side.fork[k] && cudaEventCreateWithFlags(&c->side.fork[k], cudaEventDisableTiming) != cudaSuccess)
            return false;
        if (!c->side.join[k] && cudaEventCreateWithFlags(&c->side.join[k], cudaEventDisableTiming) != cudaSuccess)
            return false;
    }
    c->side_ok = true;
    return true;
}

static cudaError_t launch_phased(ocpf_ctx* c, PhasedLauncher k, const PhasedArgs& args, cudaStream_t st,
                                 bool graph_ok, bool mark)
{
    const SideStreams* sd = (args.opts & PH_EARLY) ? &c->side : nullptr;
    // the part marks are taken on direct launches: events recorded by a
    // replayed graph's nodes cannot be timed against each other
    const cudaEvent_t* mk = mark ? c->marks : nullptr;
    c->marked             = mark;
    if (mark) graph_ok = false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusInvalidated;
    c->last_kernels = -1;
    const LaunchTune& t = c->tune;
    if (!graph_ok || cs != cudaStreamCaptureStatusNone || c->launches++ == 0) return k(c->fc, args, t, st, mk, sd);
    if (!(c->gvalid && std::memcmp(&c->gkey, &args, sizeof(args)) == 0 &&
          std::memcmp(&c->gtune, &t, sizeof(t)) == 0 && c->gmark == mark)) {
        c->gvalid = false;
        if (!c->gs && cudaStreamCreateWithFlags(&c->gs, cudaStreamNonBlocking) != cudaSuccess)
            return k(c->fc, args, t, st, mk, sd);
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(c->gs, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return k(c->fc, args, t, st, mk, sd);
        const cudaError_t le = k(c->fc, args, t, c->gs, mk, sd);
        const cudaError_t ce = cudaStreamEndCapture(c->gs, &g);
        if (le != cudaSuccess || ce != cudaSuccess || !g) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return k(c->fc, args, t, st, mk, sd);
        }
        size_t nn = 0;
        int    nk = 0;
        if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn > 0) {
            std::vector<cudaGraphNode_t> nodes(nn);
            if (cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess)
                for (size_t i = 0; i < nn; i++) {
                    cudaGraphNodeType t;
                    if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) nk++;
                }
        }
        c->gkernels = nk;
        bool ok = false;
        if (c->gexec) {
            cudaGraphExecUpdateResultInfo info;
            ok = cudaGraphExecUpdate(c->gexec, g, &info) == cudaSuccess;
            if (!ok) {
                cudaGetLastError();
                cudaGraphExecDestroy(c->gexec);
                c->gexec = nullptr;
            }
        }
        if (!ok) ok = cudaGraphInstantiate(&c->gexec, g, cudaGraphInstantiateFlagUseNodePriority) == cudaSuccess;
        cudaGraphDestroy(g);
        if (!ok) {
            c->gexec = nullptr;
            cudaGetLastError();
            return k(c->fc, args, t, st, mk, sd);
        }
        c->gkey   = args;
        c->gtune  = t;
        c->gmark  = mark;
        c->gvalid = true;
    }
    c->last_kernels = c->gkernels;
    return cudaGraphLaunch(c->gexec, st);
}

static int launch_form(ocpf_ctx* c, int form, int64_t count, int64_t stride, const ocpf_fim_in& in,
                       const ocpf_skip& sk, const ocpf_fim_out& out, cudaStream_t st, bool timed,
                       int part = -1, FlashTail tail = FlashTail{FM_FIM, nullptr, nullptr, nullptr})
{
    if (count == 0) return OCPF_OK;
    cudaError_t e;
    if (form == OCPF_FORM_PLAIN) {
        PlainLauncher k = plain_kernel(c->fc.nc);
        if (!k) return OCPF_EUNSUPPORTED;
        const int     bs     = 128;
        const int64_t blocks = (count + bs - 1) / bs;
        if (blocks > 0x7fffffffLL) return OCPF_EINVAL;
        if (timed) cudaEventRecord(c->ev0, st);
        e               = k(c->fc, count, stride, in, sk, out, tail, (unsigned)blocks, bs, st);
        c->last_kernels = 1;
        c->marked       = false;
        if (timed) cudaEventRecord(c->ev1, st);
    } else {
        int            nd = 0;
        PhasedLauncher k  = phased_kernel(c->fc.nc, &nd);
        if (!k) return OCPF_EUNSUPPORTED;
        PhasedArgs args;
        std::memset(&args, 0, sizeof(args));  // compared bytewise as the graph's key
        args.count  = count;
        args.stride = stride;
        args.in     = in;
        args.sk     = sk;
        args.out    = out;
        args.opts   = form >= OCPF_FORM_MIXED ? PH_MIXED : 0u;
        args.mlp    = c->mlp;
        args.tail   = tail;
        if (form == OCPF_FORM_FAST && c->mlp && c->fc.learn_on) args.opts |= PH_LEARN;
        // the per-trial split schedule on the device path; the host path's
        // parts, and calls that record the part marks, keep one stream
        if (part < 0 && !c->part_timing && ensure_side(c)) {
            args.opts |= PH_EARLY;
            // and the learned round beside trials 2-3 instead of before trial 0
            if (args.opts & PH_LEARN) args.opts |= PH_DEFER;
        }
        if (part < 0) {
            const int rc = ensure_scratch(c, count);
            if (rc != OCPF_OK) return rc;
            scratch_view(c, 0, c->eq_cap, args.S, args.L);
        } else {
            // host path: scratch already sized for HOST_PARTS parts of `stride` cells
            scratch_view(c, part, stride, args.S, args.L);
        }
        if (timed) cudaEventRecord(c->ev0, st);
        e = launch_phased(c, k, args, st, part < 0, timed && part < 0 && c->part_timing);
        if (timed) cudaEventRecord(c->ev1, st);
    }
    return e == cudaSuccess ? OCPF_OK : OCPF_ECUDA;
}

extern "C" int ocpf_flash_fim(ocpf_ctx* c, int64_t ncell, const ocpf_fim_in* in, ocpf_skip* sk,
                              ocpf_fim_out* out, int form, void* stream)
{
    if (!c || ncell < 0) return OCPF_EINVAL;
    if (ncell == 0) return OCPF_OK;
    if (!fim_args_ok(c, in, sk, out)) return OCPF_EINVAL;
    if (form < OCPF_FORM_PLAIN || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    ocpf_skip s{};
    if (sk) s = *sk;
    const int rc = launch_form(c, form, ncell, ncell, *in, s, *out, (cudaStream_t)stream, true);
    c->timed     = (rc == OCPF_OK && ncell > 0);
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

extern "C" int ocpf_flash_impec(ocpf_ctx* c, int64_t ncell, const ocpf_impec_in* in, ocpf_skip* sk,
                                ocpf_impec_out* out, int form, void* stream)
{
    if (!c || ncell < 0) return OCPF_EINVAL;
    if (ncell == 0) return OCPF_OK;
    if (!in || form < OCPF_FORM_PLAIN || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    if (!in->P || !in->T || !in->Ni || !in->lastNP || !in->xij) return OCPF_EINVAL;
    if (!impec_out_ok(out) || !skip_ok(c, sk)) return OCPF_EINVAL;
    ocpf_fim_in fin{};
    fin.P      = in->P;
    fin.T      = in->T;
    fin.Ni     = in->Ni;
    fin.lastNP = in->lastNP;
    fin.xij    = in->xij;
    const ocpf_fim_out fo = impec_as_fim(*out);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    ocpf_skip s{};
    if (sk) s = *sk;
    const FlashTail tail{FM_IMPEC, out->vj, nullptr, nullptr};
    const int rc = launch_form(c, form, ncell, ncell, fin, s, fo, (cudaStream_t)stream, true, -1, tail);
    c->timed     = (rc == OCPF_OK);
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

extern "C" int ocpf_flash_fimn(ocpf_ctx* c, int64_t ncell, const ocpf_fim_in* in, ocpf_skip* sk,
                               ocpf_fim_out* out, double* res, double* resPc, int form, void* stream)
{
    if (!c || ncell < 0) return OCPF_EINVAL;
    if (ncell == 0) return OCPF_OK;
    if (!fim_args_ok(c, in, sk, out) || !out->nj || !res || !resPc) return OCPF_EINVAL;
    if (form < OCPF_FORM_PLAIN || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    ocpf_skip s{};
    if (sk) s = *sk;
    const FlashTail tail{FM_FIMN, nullptr, nullptr, nullptr, res, resPc};
    const int rc = launch_form(c, form, ncell, ncell, *in, s, *out, (cudaStream_t)stream, true, -1, tail);
    c->timed     = (rc == OCPF_OK);
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

// InitFlashFIM / InitFlashIMPEC / InitFlashFIMn: the initial-state inputs as
// the FIM input record (z in place of Ni, S for the water saturation) and the
// launch; `tail` names the entry point's extra outputs (vpore and ni are
// filled in here).
static int launch_init(ocpf_ctx* c, int64_t ncell, const ocpf_init_in* in, ocpf_skip* sk, double* Ni,
                       const ocpf_fim_out& fo, FlashTail tail, int form, void* stream)
{
    ocpf_fim_in fin{};
    fin.P  = in->P;
    fin.T  = in->T;
    fin.Ni = in->zi;
    fin.S  = in->S;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    ocpf_skip s{};
    if (sk) s = *sk;
    tail.mode |= FM_INIT;
    tail.vpore = in->Vpore;
    tail.ni    = Ni;
    const int rc = launch_form(c, form, ncell, ncell, fin, s, fo, (cudaStream_t)stream, true, -1, tail);
    c->timed     = (rc == OCPF_OK);
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

static bool init_in_ok(const ocpf_init_in* in)
{
    return in && in->P && in->T && in->S && in->Vpore && in->zi;
}

extern "C" int ocpf_init_flash_fim(ocpf_ctx* c, int64_t ncell, const ocpf_init_in* in, ocpf_skip* sk, double* Ni,
                                   ocpf_fim_out* out, int form, void* stream)
{
    if (!c || ncell < 0) return OCPF_EINVAL;
    if (ncell == 0) return OCPF_OK;
    if (form < OCPF_FORM_PLAIN || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    if (!init_in_ok(in) || !Ni || !fim_out_ok(out) || !skip_ok(c, sk)) return OCPF_EINVAL;
    return launch_init(c, ncell, in, sk, Ni, *out, FlashTail{FM_FIM, nullptr, nullptr, nullptr}, form, stream);
}

extern "C" int ocpf_init_flash_impec(ocpf_ctx* c, int64_t ncell, const ocpf_init_in* in, ocpf_skip* sk,
                                     double* Ni, ocpf_impec_out* out, int form, void* stream)
{
    if (!c || ncell < 0) return OCPF_EINVAL;
    if (ncell == 0) return OCPF_OK;
    if (form < OCPF_FORM_PLAIN || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    if (!init_in_ok(in) || !Ni || !impec_out_ok(out) || !skip_ok(c, sk)) return OCPF_EINVAL;
    return launch_init(c, ncell, in, sk, Ni, impec_as_fim(*out), FlashTail{FM_IMPEC, out->vj, nullptr, nullptr},
                       form, stream);
}

extern "C" int ocpf_init_flash_fimn(ocpf_ctx* c, int64_t ncell, const ocpf_init_in* in, ocpf_skip* sk, double* Ni,
                                    ocpf_fim_out* out, double* res, double* resPc, int form, void* stream)
{
    if (!c || ncell < 0) return OCPF_EINVAL;
    if (ncell == 0) return OCPF_OK;
    if (form < OCPF_FORM_PLAIN || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    if (!init_in_ok(in) || !Ni || !fim_out_ok(out) || !out->nj || !res || !resPc || !skip_ok(c, sk))
        return OCPF_EINVAL;
    return launch_init(c, ncell, in, sk, Ni, *out, FlashTail{FM_FIMN, nullptr, nullptr, nullptr, res, resPc}, form,
                       stream);
}

// The one-launch sequence of ocpf_flash_fim_regions, replayed from a CUDA
// graph held by the leading context while the arguments and the launch
// shape stay the same (as launch_phased does for one region).
static cudaError_t launch_multi(ocpf_ctx* c, const MultiFluid& MF, const MultiArgs& M, cudaStream_t st)
{
    const LaunchTune&       t  = c->tune;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusInvalidated;
    c->last_kernels = -1;
    if (cs != cudaStreamCaptureStatusNone) return launch_phased_multi(MF, M, t, st);
    const bool same = c->mgexec && c->mgkey && std::memcmp(c->mgkey, &M, sizeof(M)) == 0 &&
                      std::memcmp(&c->mgtune, &t, sizeof(t)) == 0;
    if (!same) {
        if (!c->mgkey) {
            c->mgkey = new (std::nothrow) MultiArgs;
            if (!c->mgkey) return launch_phased_multi(MF, M, t, st);
            std::memset(c->mgkey, 0, sizeof(MultiArgs));
            // the first call launches directly (it also sets up each kernel)
            std::memcpy(c->mgkey, &M, sizeof(M));
            c->mgtune = t;
            return launch_phased_multi(MF, M, t, st);
        }
        if (!c->gs && cudaStreamCreateWithFlags(&c->gs, cudaStreamNonBlocking) != cudaSuccess)
            return launch_phased_multi(MF, M, t, st);
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(c->gs, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return launch_phased_multi(MF, M, t, st);
        const cudaError_t le = launch_phased_multi(MF, M, t, c->gs);
        const cudaError_t ce = cudaStreamEndCapture(c->gs, &g);
        if (le != cudaSuccess || ce != cudaSuccess || !g) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return launch_phased_multi(MF, M, t, st);
        }
        size_t nn = 0;
        int    nk = 0;
        if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn > 0) {
            std::vector<cudaGraphNode_t> nodes(nn);
            if (cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess)
                for (size_t i = 0; i < nn; i++) {
                    cudaGraphNodeType ty;
                    if (cudaGraphNodeGetType(nodes[i], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) nk++;
                }
        }
        if (c->mgexec) cudaGraphExecDestroy(c->mgexec);
        c->mgexec = nullptr;
        const bool ok = cudaGraphInstantiate(&c->mgexec, g, 0) == cudaSuccess;
        cudaGraphDestroy(g);
        if (!ok) {
            c->mgexec = nullptr;
            cudaGetLastError();
            return launch_phased_multi(MF, M, t, st);
        }
        std::memcpy(c->mgkey, &M, sizeof(M));
        c->mgtune    = t;
        c->mgkernels = nk;
    }
    c->last_kernels = c->mgkernels;
    return cudaGraphLaunch(c->mgexec, st);
}

static bool multi_nc_ok(int nc) { return nc == 3 || nc == 6 || nc == 9 || nc == 12; }

// Every non-empty region in one launch sequence (OCPF_SCHED_ONE_LAUNCH).
static int regions_one_launch(int nreg, ocpf_ctx* const* ctx, const int64_t* ncell, const ocpf_fim_in* in,
                              ocpf_skip* sk, ocpf_fim_out* out, int form, cudaStream_t st)
{
    MultiFluid* MF = new (std::nothrow) MultiFluid;
    if (!MF) return OCPF_ENOMEM;
    MultiArgs M;
    std::memset(&M, 0, sizeof(M));  // compared bytewise as the graph's key
    int rc = OCPF_OK, n = 0;
    for (int r = 0; r < nreg && rc == OCPF_OK; r++) {
        if (ncell[r] == 0) continue;
        ocpf_ctx* c = ctx[r];
        rc          = ensure_scratch(c, ncell[r]);
        if (rc != OCPF_OK) break;
        PhasedArgs& a = M.a[n];
        a.count  = ncell[r];
        a.stride = ncell[r];
        a.in     = in[r];
        a.sk     = sk ? sk[r] : ocpf_skip{};
        a.out    = out[r];
        a.opts   = form >= OCPF_FORM_MIXED ? PH_MIXED : 0u;
        a.mlp    = c->mlp;
        a.tail   = FlashTail{FM_FIM, nullptr, nullptr, nullptr};
        if (form == OCPF_FORM_FAST && c->mlp && c->fc.learn_on) a.opts |= PH_LEARN;
        scratch_view(c, 0, c->eq_cap, a.S, a.L);
        MF->F[n] = c->fc;
        M.nc[n]  = c->fc.nc;
        n++;
    }
    if (rc == OCPF_OK && n > 0) {
        M.n = n;
        for (int r = 0; r < n; r++) {
            M.a[r].vpart  = r;
            M.a[r].vparts = n;
        }
        if (launch_multi(ctx[0], *MF, M, st) != cudaSuccess) rc = OCPF_ECUDA;
    }
    delete MF;
    return rc;
}

// One launch sequence per region on the regions' own streams (OCPF_SCHED_STREAMS).
static int regions_streams(int nreg, ocpf_ctx* const* ctx, const int64_t* ncell, const ocpf_fim_in* in,
                           ocpf_skip* sk, ocpf_fim_out* out, int form, cudaStream_t stream)
{
    int rc = OCPF_OK;
    for (int r = 0; r < nreg && rc == OCPF_OK; r++) {
        ocpf_ctx* c = ctx[r];
        if (!c->rs && cudaStreamCreateWithFlags(&c->rs, cudaStreamNonBlocking) != cudaSuccess) rc = OCPF_ECUDA;
        if (rc == OCPF_OK && !c->evf && cudaEventCreateWithFlags(&c->evf, cudaEventDisableTiming) != cudaSuccess)
            rc = OCPF_ECUDA;
        if (rc == OCPF_OK && !c->evj && cudaEventCreateWithFlags(&c->evj, cudaEventDisableTiming) != cudaSuccess)
            rc = OCPF_ECUDA;
    }
    // fork: every region's stream starts after the work already on `stream`
    if (rc == OCPF_OK && cudaEventRecord(ctx[0]->evf, stream) != cudaSuccess) rc = OCPF_ECUDA;
    for (int r = 0; r < nreg && rc == OCPF_OK; r++) {
        ocpf_ctx* c = ctx[r];
        if (cudaStreamWaitEvent(c->rs, ctx[0]->evf, 0) != cudaSuccess) {
            rc = OCPF_ECUDA;
            break;
        }
        ocpf_skip s{};
        if (sk) s = sk[r];
        if (ncell[r] > 0) rc = launch_form(c, form, ncell[r], ncell[r], in[r], s, out[r], c->rs, false);
        c->timed = false;
        // join: `stream` continues after every region
        if (rc == OCPF_OK && (cudaEventRecord(c->evj, c->rs) != cudaSuccess ||
                              cudaStreamWaitEvent(stream, c->evj, 0) != cudaSuccess))
            rc = OCPF_ECUDA;
    }
    return rc;
}

static int regions_check(int nreg, ocpf_ctx* const* ctx, const int64_t* ncell, const ocpf_fim_in* in,
                         const ocpf_skip* sk, const ocpf_fim_out* out, int form)
{
    if (nreg < 0) return OCPF_EINVAL;
    if (nreg == 0) return OCPF_OK;
    if (!ctx || !ncell || !in || !out) return OCPF_EINVAL;
    if (form < OCPF_FORM_PLAIN || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    for (int r = 0; r < nreg; r++) {
        if (!ctx[r] || ncell[r] < 0 || ctx[r]->device != ctx[0]->device) return OCPF_EINVAL;
        for (int q = 0; q < r; q++)
            if (ctx[q] == ctx[r]) return OCPF_EINVAL;  // one context owns one scratch and stream
        if (ncell[r] > 0 && !fim_args_ok(ctx[r], &in[r], sk ? &sk[r] : nullptr, &out[r])) return OCPF_EINVAL;
    }
    return OCPF_OK;
}

static bool one_launch_ok(int nreg, ocpf_ctx* const* ctx, int form)
{
    if (form == OCPF_FORM_PLAIN || nreg > MULTI_MAX || ctx[0]->sched != OCPF_SCHED_ONE_LAUNCH) return false;
    for (int r = 0; r < nreg; r++)
        if (!multi_nc_ok(ctx[r]->fc.nc)) return false;
    return true;
}

extern "C" int ocpf_flash_fim_regions(int nreg, ocpf_ctx* const* ctx, const int64_t* ncell, const ocpf_fim_in* in,
                                      ocpf_skip* sk, ocpf_fim_out* out, int form, void* stream)
{
    int rc = regions_check(nreg, ctx, ncell, in, sk, out, form);
    if (rc != OCPF_OK || nreg == 0) return rc;
    int prev = 0;
    cudaGetDevice(&prev);
    const int dev = ctx[0]->device;
    if (prev != dev) cudaSetDevice(dev);
    if (one_launch_ok(nreg, ctx, form))
        rc = regions_one_launch(nreg, ctx, ncell, in, sk, out, form, (cudaStream_t)stream);
    else
        rc = regions_streams(nreg, ctx, ncell, in, sk, out, form, (cudaStream_t)stream);
    for (int r = 0; r < nreg; r++) ctx[r]->timed = false;
    if (prev != dev) cudaSetDevice(prev);
    return rc;
}

// ------------------------------------------------------------------ tuning
extern "C" int ocpf_get_tuning(const ocpf_ctx* c, ocpf_tuning* t)
{
    if (!c || !t) return OCPF_EINVAL;
    t->block        = c->tune.block;
    t->persist_pct  = c->tune.persist_pct;
    t->slow_threads = c->tune.slow_threads;
    t->schedule     = c->sched;
    t->ms           = c->tune_ms;
    t->pad          = 0;
    return OCPF_OK;
}

extern "C" int ocpf_set_tuning(ocpf_ctx* c, const ocpf_tuning* t)
{
    if (!c || !t) return OCPF_EINVAL;
    if ((t->block != 64 && t->block != 128) || t->persist_pct < 1 || t->persist_pct > 100 ||
        (t->slow_threads != 0 && t->slow_threads != 1) ||
        (t->schedule != OCPF_SCHED_ONE_LAUNCH && t->schedule != OCPF_SCHED_STREAMS))
        return OCPF_EINVAL;
    c->tune    = LaunchTune{t->block, t->persist_pct, t->slow_threads, 0};
    c->sched   = t->schedule;
    c->tune_ms = t->ms;
    return OCPF_OK;
}

extern "C" int ocpf_last_launch_count(ocpf_ctx* c, int* n)
{
    if (!c || !n) return OCPF_EINVAL;
    *n = c->last_kernels;
    return OCPF_OK;
}

extern "C" int ocpf_set_part_timing(ocpf_ctx* c, int on)
{
    if (!c) return OCPF_EINVAL;
    c->part_timing = on != 0;
    return OCPF_OK;
}

extern "C" int ocpf_last_phase_ms(ocpf_ctx* c, float* ms)
{
    if (!c || !ms) return OCPF_EINVAL;
    ms[0] = ms[1] = ms[2] = 0;
    if (!c->timed || !c->marked) return OCPF_OK;
    if (cudaEventSynchronize(c->ev1) != cudaSuccess) return OCPF_ECUDA;
    if (cudaEventElapsedTime(&ms[0], c->ev0, c->marks[0]) != cudaSuccess ||
        cudaEventElapsedTime(&ms[1], c->marks[0], c->marks[1]) != cudaSuccess ||
        cudaEventElapsedTime(&ms[2], c->marks[1], c->ev1) != cudaSuccess)
        return OCPF_ECUDA;
    return OCPF_OK;
}

extern "C" int ocpf_last_kernel_ms(ocpf_ctx* c, float* ms)
{
    if (!c || !ms) return OCPF_EINVAL;
    if (!c->timed) {
        *ms = 0;
        return OCPF_OK;
    }
    if (cudaEventSynchronize(c->ev1) != cudaSuccess) return OCPF_ECUDA;
    return cudaEventElapsedTime(ms, c->ev0, c->ev1) == cudaSuccess ? OCPF_OK : OCPF_ECUDA;
}

// ------------------------------------------------------------ host path

namespace {

// Field counts of each SoA array group, per cell.
struct Layout {
    int nc, ncom, ncol;
    // doubles per cell
    int in_d() const { return 2 + ncom + NPH + NPH * ncom; }             // P, T, Ni, S, xij
    int sk_d() const { return 3 + nc; }                                  // minEig, P, T, z
    int out_d() const
    {
        return NPH + 3 + ncom + 6 * NPH + 4 * NPH * ncom + NPH * ncol * ncol + NPH + 1;  // + nj, ePEC
    }
    int u32() const { return 1 + 1 + NPH + 1 + NPH + NPH + 1 + 5; }   // lastNP, phaseNum, phaseExist,
                                                                     // bRow, pSder, pVnum, skflag, iters
    int u16() const { return 1; }
    int u8() const { return 1; }
    size_t bytes_per_cell() const
    {
        return (size_t)(in_d() + sk_d() + out_d()) * 8 + (size_t)u32() * 4 + u16() * 2 + u8();
    }
};

// Bytes of one staging buffer, rounded up to 256 so that the second buffer
// (and every array carved from it) stays aligned.
inline size_t stage_stride(size_t per_cell, int64_t cap) { return ((per_cell * (size_t)cap + 255) / 256) * 256; }

// Carves per-chunk device views out of one staging block (stride = cap).
struct Views {
    ocpf_fim_in  in;
    ocpf_skip    sk;
    ocpf_fim_out out;
};

Views carve(void* base, int64_t cap, const Layout& L, const ocpf_skip* hsk, const ocpf_fim_out* ho)
{
    Views   v{};
    char*   p   = (char*)base;
    auto    D   = [&](int nf) { double* r = (double*)p; p += (size_t)nf * cap * 8; return r; };
    auto    U32 = [&](int nf) { uint32_t* r = (uint32_t*)p; p += (size_t)nf * cap * 4; return r; };
    v.in.P          = D(1);
    v.in.T          = D(1);
    v.in.Ni         = D(L.ncom);
    v.in.S          = D(NPH);
    v.in.xij        = D(NPH * L.ncom);
    v.sk.minEig     = D(1);
    v.sk.P          = D(1);
    v.sk.T          = D(1);
    v.sk.z          = D(L.nc);
    v.out.S         = D(NPH);
    v.out.Nt        = D(1);
    v.out.vf        = D(1);
    v.out.vfP       = D(1);
    v.out.vfi       = D(L.ncom);
    v.out.rho       = D(NPH);
    v.out.xi        = D(NPH);
    v.out.mu        = D(NPH);
    v.out.rhoP      = D(NPH);
    v.out.xiP       = D(NPH);
    v.out.muP       = D(NPH);
    v.out.xij       = D(NPH * L.ncom);
    v.out.rhox      = D(NPH * L.ncom);
    v.out.xix       = D(NPH * L.ncom);
    v.out.mux       = D(NPH * L.ncom);
    v.out.dSec_dPri = D(NPH * L.ncol * L.ncol);
    v.out.nj        = D(NPH);
    v.out.ePEC      = D(1);
    v.in.lastNP     = U32(1);
    v.out.phaseNum  = U32(1);
    v.out.phaseExist = U32(NPH);
    v.out.bRowSizedSdP = U32(1);
    v.out.pSderExist = U32(NPH);
    v.out.pVnumCom  = U32(NPH);
    v.sk.flag       = U32(1);
    v.out.iters     = (int32_t*)U32(5);
    v.out.status    = (uint16_t*)p;
    p += (size_t)cap * 2;
    v.out.ftype = (uint8_t*)p;
    p += (size_t)cap;
    if (!hsk) v.sk = ocpf_skip{};
    if (!ho->nj) v.out.nj = nullptr;
    if (!ho->ePEC) v.out.ePEC = nullptr;
    if (!ho->iters) v.out.iters = nullptr;
    if (!ho->status) v.out.status = nullptr;
    if (!ho->ftype) v.out.ftype = nullptr;
    return v;
}

// Copies nf fields of `esz`-byte elements for cells [c0, c0+cnt) between a
// host SoA array (stride ncell) and a staging array (stride cap).
inline cudaError_t copy_fields(void* dst, const void* src, int nf, size_t esz, int64_t c0,
                               int64_t cnt, int64_t ncell, int64_t cap, bool h2d, cudaStream_t st)
{
    if (!dst || !src || cnt == 0) return cudaSuccess;
    if (h2d)
        return cudaMemcpy2DAsync(dst, cap * esz, (const char*)src + c0 * esz, ncell * esz, cnt * esz,
                                 nf, cudaMemcpyHostToDevice, st);
    return cudaMemcpy2DAsync((char*)dst + c0 * esz, ncell * esz, src, cap * esz, cnt * esz, nf,
                             cudaMemcpyDeviceToHost, st);
}

}  // namespace

extern "C" int ocpf_flash_fim_host(ocpf_ctx* c, int64_t ncell, const ocpf_fim_in* in, ocpf_skip* sk,
                                   ocpf_fim_out* out, int form)
{
    if (!c || ncell < 0) return OCPF_EINVAL;
    if (ncell == 0) return OCPF_OK;
    if (!fim_args_ok(c, in, sk, out)) return OCPF_EINVAL;
    if (form < OCPF_FORM_PLAIN || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    int rc = OCPF_OK;
    Layout L{c->fc.nc, c->fc.nc + 1, c->fc.nc + 2};
    const int64_t chunk = std::min<int64_t>(ncell, 131072);
    const size_t  per   = L.bytes_per_cell();
    if (c->stage_cap < chunk) {
        if (c->stage) cudaFree(c->stage);
        c->stage     = nullptr;
        c->stage_cap = 0;
        if (cudaMalloc(&c->stage, HOST_PARTS * stage_stride(per, chunk)) != cudaSuccess) {
            if (prev != c->device) cudaSetDevice(prev);
            return OCPF_ENOMEM;
        }
        c->stage_cap = chunk;
    }
    for (auto& s : c->hs)
        if (!s) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    for (auto& ev : c->hdone)
        if (!ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    const int64_t cap = c->stage_cap;
    if (form != OCPF_FORM_PLAIN) {
        const int r2 = ensure_scratch(c, cap, HOST_PARTS);
        if (r2 != OCPF_OK) {
            if (prev != c->device) cudaSetDevice(prev);
            return r2;
        }
    }
    Views V[HOST_PARTS];
    for (int b = 0; b < HOST_PARTS; b++) V[b] = carve((char*)c->stage + b * stage_stride(per, cap), cap, L, sk, out);
    const bool use_sk = c->fc.use_skip != 0;
    // Each chunk goes to a part whose previous chunk has been copied out
    // (first every part once, then whichever finishes first), so a chunk
    // that holds a long restart chain keeps only its own part busy instead
    // of also holding back the chunks dealt to the same stream after it.
    int nused = 0;
    auto next_part = [&]() -> int {
        if (nused < HOST_PARTS) return nused++;
        for (;;) {
            for (int b = 0; b < HOST_PARTS; b++) {
                const cudaError_t q = cudaEventQuery(c->hdone[b]);
                if (q == cudaSuccess) return b;
                if (q != cudaErrorNotReady) return -1;
            }
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    };
    for (int64_t c0 = 0; c0 < ncell && rc == OCPF_OK; c0 += cap) {
        const int bidx = next_part();
        if (bidx < 0) {
            rc = OCPF_ECUDA;
            break;
        }
        const int64_t cnt = std::min<int64_t>(cap, ncell - c0);
        cudaStream_t  st  = c->hs[bidx];
        const Views&  v   = V[bidx];
        cudaError_t   e   = cudaSuccess;
        auto H = [&](void* d, const void* s, int nf, size_t esz) {
            if (e == cudaSuccess) e = copy_fields(d, s, nf, esz, c0, cnt, ncell, cap, true, st);
        };
        auto D = [&](void* h, const void* d, int nf, size_t esz) {
            if (e == cudaSuccess && h && d) e = copy_fields(h, d, nf, esz, c0, cnt, ncell, cap, false, st);
        };
        H((void*)v.in.P, in->P, 1, 8);
        H((void*)v.in.T, in->T, 1, 8);
        H((void*)v.in.Ni, in->Ni, L.ncom, 8);
        H((void*)v.in.S, in->S, NPH, 8);
        H((void*)v.in.xij, in->xij, NPH * L.ncom, 8);
        H((void*)v.in.lastNP, in->lastNP, 1, 4);
        // outputs of absent phases are left untouched: stage the caller's values
        H(v.out.rho, out->rho, NPH, 8);
        H(v.out.xi, out->xi, NPH, 8);
        H(v.out.mu, out->mu, NPH, 8);
        H(v.out.rhoP, out->rhoP, NPH, 8);
        H(v.out.xiP, out->xiP, NPH, 8);
        H(v.out.muP, out->muP, NPH, 8);
        H(v.out.xij, out->xij, NPH * L.ncom, 8);
        H(v.out.rhox, out->rhox, NPH * L.ncom, 8);
        H(v.out.xix, out->xix, NPH * L.ncom, 8);
        H(v.out.mux, out->mux, NPH * L.ncom, 8);
        if (out->nj) H(v.out.nj, out->nj, NPH, 8);
        if (use_sk) {
            H(v.sk.flag, sk->flag, 1, 4);
            H(v.sk.minEig, sk->minEig, 1, 8);
            H(v.sk.P, sk->P, 1, 8);
            H(v.sk.T, sk->T, 1, 8);
            H(v.sk.z, sk->z, L.nc, 8);
        }
        if (e != cudaSuccess) {
            rc = OCPF_ECUDA;
            break;
        }
        rc = launch_form(c, form, cnt, cap, v.in, v.sk, v.out, st, false, bidx);
        if (rc != OCPF_OK) break;
        D(out->phaseNum, v.out.phaseNum, 1, 4);
        D(out->phaseExist, v.out.phaseExist, NPH, 4);
        D(out->S, v.out.S, NPH, 8);
        D(out->Nt, v.out.Nt, 1, 8);
        D(out->vf, v.out.vf, 1, 8);
        D(out->vfP, v.out.vfP, 1, 8);
        D(out->vfi, v.out.vfi, L.ncom, 8);
        D(out->rho, v.out.rho, NPH, 8);
        D(out->xi, v.out.xi, NPH, 8);
        D(out->mu, v.out.mu, NPH, 8);
        D(out->rhoP, v.out.rhoP, NPH, 8);
        D(out->xiP, v.out.xiP, NPH, 8);
        D(out->muP, v.out.muP, NPH, 8);
        D(out->xij, v.out.xij, NPH * L.ncom, 8);
        D(out->rhox, v.out.rhox, NPH * L.ncom, 8);
        D(out->xix, v.out.xix, NPH * L.ncom, 8);
        D(out->mux, v.out.mux, NPH * L.ncom, 8);
        D(out->dSec_dPri, v.out.dSec_dPri, NPH * L.ncol * L.ncol, 8);
        D(out->bRowSizedSdP, v.out.bRowSizedSdP, 1, 4);
        D(out->pSderExist, v.out.pSderExist, NPH, 4);
        D(out->pVnumCom, v.out.pVnumCom, NPH, 4);
        D(out->nj, v.out.nj, NPH, 8);
        D(out->ePEC, v.out.ePEC, 1, 8);
        D(out->ftype, v.out.ftype, 1, 1);
        D(out->iters, v.out.iters, 5, 4);
        D(out->status, v.out.status, 1, 2);
        if (use_sk) {
            D(sk->flag, v.sk.flag, 1, 4);
            D(sk->minEig, v.sk.minEig, 1, 8);
            D(sk->P, v.sk.P, 1, 8);
            D(sk->T, v.sk.T, 1, 8);
            D(sk->z, v.sk.z, L.nc, 8);
        }
        if (e == cudaSuccess) e = cudaEventRecord(c->hdone[bidx], st);
        if (e != cudaSuccess) rc = OCPF_ECUDA;
    }
    for (auto& s : c->hs)
        if (cudaStreamSynchronize(s) != cudaSuccess) rc = OCPF_ECUDA;
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

extern "C" int ocpf_reserve(ocpf_ctx* c, int64_t ncell)
{
    if (!c || ncell < 0) return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    const int rc = ensure_scratch(c, ncell);
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

extern "C" int ocpf_set_initializer(ocpf_ctx* c, const float* params, const float* in_mean, const float* in_scale,
                                    float confidence)
{
    if (!c || !params || !in_mean || !in_scale || !(confidence > 0.5f) || !(confidence < 1.0f)) return OCPF_EINVAL;
    const int nf = c->fc.nc + 2;
    for (int f = 0; f < nf; f++)
        if (!(in_scale[f] > 0.f) || !std::isfinite(in_mean[f])) return OCPF_EINVAL;
    const int np = ocpf_mlp_param_count();
    for (int i = 0; i < np; i++)
        if (!std::isfinite(params[i])) return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    int rc = OCPF_OK;
    if (!c->mlp && cudaMalloc(&c->mlp, sizeof(float) * np) != cudaSuccess) {
        c->mlp = nullptr;
        rc     = OCPF_ENOMEM;
    }
    if (rc == OCPF_OK && cudaMemcpy(c->mlp, params, sizeof(float) * np, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = OCPF_ECUDA;
    if (rc == OCPF_OK) {
        for (int f = 0; f < nf; f++) {
            c->fc.lin_mean[f]  = in_mean[f];
            c->fc.lin_scale[f] = in_scale[f];
        }
        c->fc.learn_conf = confidence;
        c->fc.learn_on   = 1;
        c->gvalid        = false;  // the constants a captured graph holds changed
    }
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

// ------------------------------------------------------------ subsets

namespace {

// The arrays one gather or scatter moves: `rows` fields of `esz`-byte
// elements between a full SoA array (stride ncell) and a compact one
// (stride nsub), for the cells idx[0..nsub).
constexpr int SUB_MAX = 48;
struct SubTable {
    int            n;
    int64_t        nsub, ncell;
    const int64_t* idx;
    char*          full[SUB_MAX];
    char*          comp[SUB_MAX];
    int            rows[SUB_MAX];
    int            esz[SUB_MAX];
    // cpt: carved from the context's own copies, so writable even where the
    // view that holds it is const
    void add(const void* f, const void* cpt, int r, int e)
    {
        if (!f || !cpt || n >= SUB_MAX) return;
        full[n] = (char*)f;
        comp[n] = (char*)cpt;
        rows[n] = r;
        esz[n]  = e;
        n++;
    }
};

template <typename T>
__device__ __forceinline__ void sub_move(char* full, char* comp, int64_t fo, int64_t co, bool gather)
{
    if (gather)
        ((T*)comp)[co] = ((const T*)full)[fo];
    else
        ((T*)full)[fo] = ((const T*)comp)[co];
}

// blockIdx.y: the array; x: grid-stride over its rows x nsub elements.
// An index outside [0, ncell) names no cell: the gather fills its compact
// slot with zeros (a flash of zero moles ends at once with a non-finite
// status, instead of running on whatever the slot held before) and the
// scatter leaves the full arrays alone.
__global__ void k_subset_copy(const __grid_constant__ SubTable t, bool gather)
{
    const int     a     = blockIdx.y;
    const int64_t total = (int64_t)t.rows[a] * t.nsub;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / t.nsub, cc = e - r * t.nsub;
        const int64_t n = t.idx[cc];
        const int64_t co = r * t.nsub + cc;
        if (n < 0 || n >= t.ncell) {
            if (gather) {
                switch (t.esz[a]) {
                    case 8: ((uint64_t*)t.comp[a])[co] = 0; break;
                    case 4: ((uint32_t*)t.comp[a])[co] = 0; break;
                    case 2: ((uint16_t*)t.comp[a])[co] = 0; break;
                    default: ((uint8_t*)t.comp[a])[co] = 0; break;
                }
            }
            continue;
        }
        const int64_t fo = r * t.ncell + n;
        switch (t.esz[a]) {
            case 8: sub_move<uint64_t>(t.full[a], t.comp[a], fo, co, gather); break;
            case 4: sub_move<uint32_t>(t.full[a], t.comp[a], fo, co, gather); break;
            case 2: sub_move<uint16_t>(t.full[a], t.comp[a], fo, co, gather); break;
            default: sub_move<uint8_t>(t.full[a], t.comp[a], fo, co, gather); break;
        }
    }
}

cudaError_t subset_copy(const SubTable& t, bool gather, int device, cudaStream_t st)
{
    if (t.n == 0 || t.nsub == 0) return cudaSuccess;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0) sms = 1;
    int64_t rows = 0;
    for (int a = 0; a < t.n; a++) rows = rows > t.rows[a] ? rows : t.rows[a];
    const int64_t want = (rows * t.nsub + 255) / 256;
    dim3 grid((unsigned)(want < (int64_t)sms * 4 ? want : (int64_t)sms * 4), t.n);
    k_subset_copy<<<grid, 256, 0, st>>>(t, gather);
    return cudaGetLastError();
}

// The output arrays of a FIM record as table entries, full -> compact.
void add_outputs(SubTable& t, const Layout& L, const ocpf_fim_out& f, const ocpf_fim_out& cpt)
{
    const int nph = NPH, pc = NPH * L.ncom;
    t.add(f.phaseNum, cpt.phaseNum, 1, 4);
    t.add(f.phaseExist, cpt.phaseExist, nph, 4);
    t.add(f.S, cpt.S, nph, 8);
    t.add(f.Nt, cpt.Nt, 1, 8);
    t.add(f.vf, cpt.vf, 1, 8);
    t.add(f.vfP, cpt.vfP, 1, 8);
    t.add(f.vfi, cpt.vfi, L.ncom, 8);
    t.add(f.rho, cpt.rho, nph, 8);
    t.add(f.xi, cpt.xi, nph, 8);
    t.add(f.mu, cpt.mu, nph, 8);
    t.add(f.rhoP, cpt.rhoP, nph, 8);
    t.add(f.xiP, cpt.xiP, nph, 8);
    t.add(f.muP, cpt.muP, nph, 8);
    t.add(f.xij, cpt.xij, pc, 8);
    t.add(f.rhox, cpt.rhox, pc, 8);
    t.add(f.xix, cpt.xix, pc, 8);
    t.add(f.mux, cpt.mux, pc, 8);
    t.add(f.dSec_dPri, cpt.dSec_dPri, NPH * L.ncol * L.ncol, 8);
    t.add(f.bRowSizedSdP, cpt.bRowSizedSdP, 1, 4);
    t.add(f.pSderExist, cpt.pSderExist, nph, 4);
    t.add(f.pVnumCom, cpt.pVnumCom, nph, 4);
    t.add(f.nj, cpt.nj, nph, 8);
    t.add(f.ePEC, cpt.ePEC, 1, 8);
    t.add(f.ftype, cpt.ftype, 1, 1);
    t.add(f.iters, cpt.iters, 5, 4);
    t.add(f.status, cpt.status, 1, 2);
}

void add_skip(SubTable& t, const Layout& L, const ocpf_skip& f, const ocpf_skip& cpt)
{
    t.add(f.flag, cpt.flag, 1, 4);
    t.add(f.minEig, cpt.minEig, 1, 8);
    t.add(f.P, cpt.P, 1, 8);
    t.add(f.T, cpt.T, 1, 8);
    t.add(f.z, cpt.z, L.nc, 8);
}

// A compact pointer only where the caller passed the array.
template <typename T>
void keep_if(T*& cpt, const void* full)
{
    if (!full) cpt = nullptr;
}

// The flash of the cells idx[0..nsub) of full arrays of ncell cells: the
// listed cells' inputs, outputs and skip cache are gathered into compact
// copies (the outputs too, so that what the flash leaves untouched -- the
// outputs of absent phases -- goes back unchanged), the chosen form runs on
// the copies, and the outputs and the skip cache are scattered back.
int flash_subset(ocpf_ctx* c, int64_t nsub, const int64_t* idx, int64_t ncell, const ocpf_fim_in& in,
                 const ocpf_skip* sk, const ocpf_fim_out& out, double* vj, FlashTail tail, int form,
                 cudaStream_t st)
{
    const Layout L{c->fc.nc, c->fc.nc + 1, c->fc.nc + 2};
    const size_t body = stage_stride(L.bytes_per_cell(), nsub);
    const size_t need = body + stage_stride((size_t)NPH * 8, nsub);
    if (c->sub_cap < nsub || !c->sub) {
        if (c->sub) {
            cudaDeviceSynchronize();  // queued work may still read the old copies
            cudaFree(c->sub);
        }
        c->sub     = nullptr;
        c->sub_cap = 0;
        c->gvalid  = false;
        if (cudaMalloc(&c->sub, need) != cudaSuccess) return OCPF_ENOMEM;
        c->sub_cap = nsub;
    }
    Views v = carve(c->sub, nsub, L, sk, &out);
    keep_if(v.in.S, in.S);
    keep_if(v.in.lastNP, in.lastNP);
    keep_if(v.in.xij, in.xij);
    ocpf_fim_out& o = v.out;
    keep_if(o.rhoP, out.rhoP);
    keep_if(o.xiP, out.xiP);
    keep_if(o.muP, out.muP);
    keep_if(o.rhox, out.rhox);
    keep_if(o.xix, out.xix);
    keep_if(o.mux, out.mux);
    keep_if(o.dSec_dPri, out.dSec_dPri);
    keep_if(o.bRowSizedSdP, out.bRowSizedSdP);
    keep_if(o.pSderExist, out.pSderExist);
    keep_if(o.pVnumCom, out.pVnumCom);
    double* vjc = vj ? (double*)((char*)c->sub + body) : nullptr;
    SubTable gin{}, gout{};
    gin.nsub = gout.nsub = nsub;
    gin.ncell = gout.ncell = ncell;
    gin.idx = gout.idx = idx;
    gin.add(in.P, v.in.P, 1, 8);
    gin.add(in.T, v.in.T, 1, 8);
    gin.add(in.Ni, v.in.Ni, L.ncom, 8);
    gin.add(in.S, v.in.S, NPH, 8);
    gin.add(in.lastNP, v.in.lastNP, 1, 4);
    gin.add(in.xij, v.in.xij, NPH * L.ncom, 8);
    add_outputs(gout, L, out, o);
    if (sk) add_skip(gout, L, *sk, v.sk);
    gout.add(vj, vjc, NPH, 8);
    if (subset_copy(gin, true, c->device, st) != cudaSuccess || subset_copy(gout, true, c->device, st) != cudaSuccess)
        return OCPF_ECUDA;
    tail.vj  = vjc;
    int rc   = launch_form(c, form, nsub, nsub, v.in, v.sk, o, st, true, -1, tail);
    c->timed = (rc == OCPF_OK);
    if (rc == OCPF_OK && subset_copy(gout, false, c->device, st) != cudaSuccess) rc = OCPF_ECUDA;
    return rc;
}

}  // namespace

extern "C" int ocpf_flash_fim_subset(ocpf_ctx* c, int64_t nsub, const int64_t* idx, int64_t ncell,
                                     const ocpf_fim_in* in, ocpf_skip* sk, ocpf_fim_out* out, int form,
                                     void* stream)
{
    if (!c || nsub < 0 || ncell < 0 || nsub > ncell) return OCPF_EINVAL;
    if (nsub == 0) return OCPF_OK;
    if (!idx || !fim_args_ok(c, in, sk, out)) return OCPF_EINVAL;
    if (form < OCPF_FORM_PLAIN || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    const int rc = flash_subset(c, nsub, idx, ncell, *in, sk, *out, nullptr,
                                FlashTail{FM_FIM, nullptr, nullptr, nullptr}, form, (cudaStream_t)stream);
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

extern "C" int ocpf_flash_impec_subset(ocpf_ctx* c, int64_t nsub, const int64_t* idx, int64_t ncell,
                                       const ocpf_impec_in* in, ocpf_skip* sk, ocpf_impec_out* out, int form,
                                       void* stream)
{
    if (!c || nsub < 0 || ncell < 0 || nsub > ncell) return OCPF_EINVAL;
    if (nsub == 0) return OCPF_OK;
    if (!idx || !in || form < OCPF_FORM_PLAIN || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    if (!in->P || !in->T || !in->Ni || !in->lastNP || !in->xij) return OCPF_EINVAL;
    if (!impec_out_ok(out) || !skip_ok(c, sk)) return OCPF_EINVAL;
    ocpf_fim_in fin{};
    fin.P      = in->P;
    fin.T      = in->T;
    fin.Ni     = in->Ni;
    fin.lastNP = in->lastNP;
    fin.xij    = in->xij;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    const int rc = flash_subset(c, nsub, idx, ncell, fin, sk, impec_as_fim(*out), out->vj,
                                FlashTail{FM_IMPEC, nullptr, nullptr, nullptr}, form, (cudaStream_t)stream);
    if (prev != c->device) cudaSetDevice(prev);
    return rc;
}

// Accessors for the library's other translation units.
namespace ocpf {
const FluidConst* ctx_fluid_const(const ocpf_ctx* c) { return &c->fc; }
int               ctx_device(const ocpf_ctx* c) { return c->device; }
bool ctx_fim_args_ok(const ocpf_ctx* c, const ocpf_fim_in* in, const ocpf_skip* sk, const ocpf_fim_out* o)
{
    return fim_args_ok(c, in, sk, o);
}
}  // namespace ocpf

extern "C" int ocpf_autotune(int nreg, ocpf_ctx* const* ctx, const int64_t* ncell, const ocpf_fim_in* in,
                             const ocpf_skip* sk, int form, int reps, void* stream, ocpf_tuning* best)
{
    if (nreg < 1 || !best || reps < 1 || form < OCPF_FORM_BATCHED || form > OCPF_FORM_FAST) return OCPF_EINVAL;
    if (!ctx || !ncell || !in) return OCPF_EINVAL;
    for (int r = 0; r < nreg; r++) {
        if (!ctx[r] || ncell[r] < 0 || ctx[r]->device != ctx[0]->device) return OCPF_EINVAL;
        for (int q = 0; q < r; q++)
            if (ctx[q] == ctx[r]) return OCPF_EINVAL;
        const ocpf_fim_in& i = in[r];
        if (ncell[r] > 0 && (!i.P || !i.T || !i.Ni || !i.S || !i.lastNP || !i.xij)) return OCPF_EINVAL;
        if (ncell[r] > 0 && !skip_ok(ctx[r], sk ? &sk[r] : nullptr)) return OCPF_EINVAL;
    }
    int prev = 0;
    cudaGetDevice(&prev);
    const int dev = ctx[0]->device;
    if (prev != dev) cudaSetDevice(dev);
    const cudaStream_t st = (cudaStream_t)stream;
    // the tuner's own copies: inputs, outputs, skip cache and its saved state
    std::vector<void*>        bufs(nreg, nullptr), skbuf(nreg, nullptr);
    std::vector<Views>        v(nreg);
    std::vector<ocpf_fim_in>  vin(nreg);
    std::vector<ocpf_skip>    vsk(nreg);
    std::vector<ocpf_fim_out> vout(nreg);
    int                       rc = OCPF_OK;
    ocpf_fim_out              all{};
    all.nj = (double*)1, all.ePEC = (double*)1, all.iters = (int32_t*)1, all.status = (uint16_t*)1,
    all.ftype = (uint8_t*)1;  // keep every diagnostic output in the views
    for (int r = 0; r < nreg && rc == OCPF_OK; r++) {
        if (ncell[r] == 0) continue;
        const Layout L{ctx[r]->fc.nc, ctx[r]->fc.nc + 1, ctx[r]->fc.nc + 2};
        const bool   has_sk = sk && sk[r].flag;
        if (cudaMalloc(&bufs[r], stage_stride(L.bytes_per_cell(), ncell[r])) != cudaSuccess) {
            rc = OCPF_ENOMEM;
            break;
        }
        v[r] = carve(bufs[r], ncell[r], L, has_sk ? &sk[r] : nullptr, &all);
        const int64_t n = ncell[r];
        const ocpf_fim_in& i = in[r];
        cudaMemcpyAsync((void*)v[r].in.P, i.P, 8 * n, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync((void*)v[r].in.T, i.T, 8 * n, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync((void*)v[r].in.Ni, i.Ni, 8 * n * L.ncom, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync((void*)v[r].in.S, i.S, 8 * n * NPH, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync((void*)v[r].in.lastNP, i.lastNP, 4 * n, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync((void*)v[r].in.xij, i.xij, 8 * n * NPH * L.ncom, cudaMemcpyDeviceToDevice, st);
        if (has_sk) {
            // the caller's cache, kept aside and restored before every run
            const size_t skb = (size_t)n * (4 + 8 * (3 + L.nc));
            if (cudaMalloc(&skbuf[r], skb) != cudaSuccess) {
                rc = OCPF_ENOMEM;
                break;
            }
            char* p = (char*)skbuf[r];
            cudaMemcpyAsync(p, sk[r].flag, 4 * n, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(p + 4 * n, sk[r].minEig, 8 * n, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(p + 12 * n, sk[r].P, 8 * n, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(p + 20 * n, sk[r].T, 8 * n, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(p + 28 * n, sk[r].z, 8 * n * L.nc, cudaMemcpyDeviceToDevice, st);
        }
        vin[r]  = v[r].in;
        vsk[r]  = v[r].sk;
        vout[r] = v[r].out;
    }
    auto restore_skip = [&]() {
        for (int r = 0; r < nreg; r++) {
            if (!skbuf[r]) continue;
            const int64_t n = ncell[r];
            const char*   p = (const char*)skbuf[r];
            cudaMemcpyAsync(vsk[r].flag, p, 4 * n, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(vsk[r].minEig, p + 4 * n, 8 * n, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(vsk[r].P, p + 12 * n, 8 * n, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(vsk[r].T, p + 20 * n, 8 * n, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(vsk[r].z, p + 28 * n, 8 * n * ctx[r]->fc.nc, cudaMemcpyDeviceToDevice, st);
        }
    };
    ocpf_tuning win{};
    win.ms = -1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rc == OCPF_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) rc = OCPF_ECUDA;
    const int blocks[2] = {128, 64}, pcts[2] = {100, 50}, slows[2] = {0, 1};
    const int nsched = nreg > 1 ? 2 : 1;
    for (int sc = 0; sc < nsched && rc == OCPF_OK; sc++)
        for (int bi = 0; bi < 2 && rc == OCPF_OK; bi++)
            for (int pi = 0; pi < 2 && rc == OCPF_OK; pi++)
                for (int si = 0; si < 2 && rc == OCPF_OK; si++) {
                    ocpf_tuning cand{blocks[bi], pcts[pi], slows[si], sc == 0 ? OCPF_SCHED_ONE_LAUNCH : OCPF_SCHED_STREAMS,
                                     0.f, 0};
                    for (int r = 0; r < nreg; r++) ocpf_set_tuning(ctx[r], &cand);
                    float bestc = 1e30f;
                    for (int k = 0; k <= reps && rc == OCPF_OK; k++) {
                        restore_skip();
                        cudaEventRecord(e0, st);
                        if (nreg == 1)
                            rc = launch_form(ctx[0], form, ncell[0], ncell[0], vin[0], vsk[0], vout[0], st, false);
                        else if (one_launch_ok(nreg, ctx, form))
                            rc = regions_one_launch(nreg, ctx, ncell, vin.data(), vsk.data(), vout.data(), form, st);
                        else
                            rc = regions_streams(nreg, ctx, ncell, vin.data(), vsk.data(), vout.data(), form, st);
                        cudaEventRecord(e1, st);
                        if (cudaEventSynchronize(e1) != cudaSuccess) rc = OCPF_ECUDA;
                        float ms = 0;
                        cudaEventElapsedTime(&ms, e0, e1);
                        if (k > 0 && ms < bestc) bestc = ms;
                    }
                    if (rc == OCPF_OK && (win.ms < 0 || bestc < win.ms)) {
                        win    = cand;
                        win.ms = bestc;
                    }
                }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamSynchronize(st);
    for (int r = 0; r < nreg; r++) {
        if (bufs[r]) cudaFree(bufs[r]);
        if (skbuf[r]) cudaFree(skbuf[r]);
    }
    if (rc == OCPF_OK) {
        for (int r = 0; r < nreg; r++) ocpf_set_tuning(ctx[r], &win);
        *best = win;
    } else {
        const ocpf_tuning def{kDefaultTune.block, kDefaultTune.persist_pct, kDefaultTune.slow_threads,
                              OCPF_SCHED_ONE_LAUNCH, 0.f, 0};
        for (int r = 0; r < nreg; r++) ocpf_set_tuning(ctx[r], &def);
    }
    if (prev != dev) cudaSetDevice(prev);
    return rc;
}
