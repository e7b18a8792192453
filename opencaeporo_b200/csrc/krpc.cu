// krpc.cu -- IsoT_FIM::CalKrPc / IsoT_IMPEC::CalKrPc for the compositional
// model's flow units (src/OCPFluidMethod.cpp:1189-1199): the default
// FlowUnit_ODGW01 (src/FlowUnit.cpp:183-349; SWOF and SGOF tables at S_w and
// S_g, Stone II oil relative permeability) and FlowUnit_ODGW02, which the
// reference selects when SOF3 is given (src/Bulk.cpp:271-279,
// src/FlowUnit.cpp:522-671; SWFN, SGFN and SOF3 tables at S_w, S_g and S_o).
// Per cell: the relative permeabilities, the capillary pressures, the phase
// pressures Pj = P + Pc_j and, for FIM, the saturation derivatives. The
// step that follows the flash: it reads the flash's S in place.
//
// One thread per cell on a grid-stride loop; every region's tables sit in
// shared memory. The kernel moves ~250 bytes per cell against ~60 FP64
// operations, so HBM bounds it. Its arithmetic is the reference's operation
// for operation with explicitly rounded intrinsics (no fused multiply-add),
// so results equal the reference's bit for bit.
#include <cstring>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "ocp_flash.h"

namespace ocpf {
namespace {

constexpr int KRPC_MAX_REG   = OCPF_KRPC_MAX_REGIONS;
constexpr int KRPC_MAX_DBL   = 6144;  // 48 KB of tables in shared memory
constexpr int KRPC_THREADS   = 256;

enum KrpcFamily : int32_t { KRPC_SWOF = 0, KRPC_SOF3 = 1 };

// Where each region's tables sit in the table buffer (column-major: column
// k of a table with nrow rows at off + k * nrow). SWOF family: w = SWOF,
// g = SGOF (4 columns). SOF3 family: w = SWFN, g = SGFN, o = SOF3 (3
// columns).
struct KrpcConst {
    int32_t nreg, total, family, pad;
    int32_t off_w[KRPC_MAX_REG], nrow_w[KRPC_MAX_REG];
    int32_t off_g[KRPC_MAX_REG], nrow_g[KRPC_MAX_REG];
    int32_t off_o[KRPC_MAX_REG], nrow_o[KRPC_MAX_REG];
};

// OCPTable::Eval_All on column 0 (src/OCPTable.cpp:47-87). The reference
// searches from the interval it found last; for a non-decreasing column the
// interval it finds is always the last node <= val, which the bisection
// here finds directly. Flat outside the table (and for NaN, which the
// reference's downward search also sends to the first row).
template <int NCOL>
__device__ __forceinline__ void eval_all(const double* t, int nrow, double val, double (&v)[NCOL],
                                         double (&s)[NCOL])
{
    if (!(val >= t[0]) || val >= t[nrow - 1]) {
        const int r = (val >= t[nrow - 1]) ? nrow - 1 : 0;
#pragma unroll
        for (int k = 0; k < NCOL; k++) {
            v[k] = t[k * nrow + r];
            s[k] = 0;
        }
        return;
    }
    int lo = 0, hi = nrow - 1;  // t[lo] <= val < t[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (t[mid] <= val)
            lo = mid;
        else
            hi = mid;
    }
    const double dx = __dsub_rn(t[lo + 1], t[lo]);
    const double u  = __dsub_rn(val, t[lo]);
#pragma unroll
    for (int k = 0; k < NCOL; k++) {
        s[k] = __ddiv_rn(__dsub_rn(t[k * nrow + lo + 1], t[k * nrow + lo]), dx);
        v[k] = __dadd_rn(t[k * nrow + lo], __dmul_rn(s[k], u));
    }
}

// FlowUnit_ODGW02 (src/FlowUnit.cpp:537-671): SWFN at S_w (krw, Pcow), SGFN
// at S_g (krg, Pcgo), SOF3 at S_o (krow, krog); kroMax is SOF3's krow at its
// last row and Swco SWFN's first saturation. The reference's two calls use
// different oil models, kept as they are: CalKrPcDeriv (FIM) Stone II with
// dKro/dS_o only (CalKro_Stone2Der, :631-652); CalKrPc (IMPEC) the default
// model (CalKro_Default, :166-177 with TINY = 1e-8, include/OCPConst.hpp).
__device__ __forceinline__ void sof3_cell(const double* st, const KrpcConst& K, int r, double So, double Sg,
                                          double Sw, bool deriv, double (&kr)[3], double (&pc)[3],
                                          double (&dkr)[9], double (&dpc)[9])
{
    const double* w = st + K.off_w[r];
    const double* g = st + K.off_g[r];
    const double* o = st + K.off_o[r];
    double        v[3], s[3];
    eval_all(w, K.nrow_w[r], Sw, v, s);
    const double krw = v[1], dkrw = s[1], pcwo = -v[2], dpcw = -s[2];
    eval_all(g, K.nrow_g[r], Sg, v, s);
    const double krg = v[1], dkrg = s[1], pcgo = v[2], dpcg = s[2];
    eval_all(o, K.nrow_o[r], So, v, s);
    const double krow = v[1], dkrow = s[1], krog = v[2], dkrog = s[2];
    const double kmax = o[2 * K.nrow_o[r] - 1];
    double       kro, dkro = 0;
    if (deriv) {
        const double a1 = __dadd_rn(__ddiv_rn(krow, kmax), krw);
        const double a2 = __dadd_rn(__ddiv_rn(krog, kmax), krg);
        kro             = __dmul_rn(kmax, __dsub_rn(__dmul_rn(a1, a2), __dadd_rn(krw, krg)));
        dkro            = __dadd_rn(__dmul_rn(dkrow, a2), __dmul_rn(dkrog, a1));
        if (kro < 0) kro = dkro = 0;
    } else {
        const double swco = w[0];
        const double tmp  = __dsub_rn(__dadd_rn(Sg, Sw), swco);
        kro = tmp <= 1e-8 ? kmax : __ddiv_rn(__dadd_rn(__dmul_rn(Sg, krog), __dmul_rn(__dsub_rn(Sw, swco), krow)), tmp);
    }
    kr[0] = kro;
    kr[1] = krg;
    kr[2] = krw;
    pc[0] = 0;
    pc[1] = pcgo;
    pc[2] = pcwo;
#pragma unroll
    for (int j = 0; j < 9; j++) dkr[j] = dpc[j] = 0;
    dkr[0] = dkro;
    dkr[4] = dkrg;
    dkr[8] = dkrw;
    dpc[4] = dpcg;
    dpc[8] = dpcw;
}

__global__ void __launch_bounds__(KRPC_THREADS) k_krpc(const __grid_constant__ KrpcConst K, const double* tab,
                                                        int64_t n, const ocpf_krpc_in in, const ocpf_krpc_out out)
{
    extern __shared__ double st[];
    for (int i = threadIdx.x; i < K.total; i += blockDim.x) st[i] = tab[i];
    __syncthreads();
    const bool deriv = out.dKr_dS != nullptr;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const int r = in.satnum ? in.satnum[c] : 0;
        double    kr[3], pc[3], dkr[9], dpc[9];
        if (r < 0 || r >= K.nreg) {
            // no such region: the reference indexes out of its flow units
#pragma unroll
            for (int j = 0; j < 3; j++) kr[j] = pc[j] = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
            for (int j = 0; j < 9; j++) dkr[j] = dpc[j] = __longlong_as_double(0x7ff8000000000000LL);
        } else if (K.family == KRPC_SOF3) {
            sof3_cell(st, K, r, in.S[c], in.S[n + c], in.S[2 * n + c], deriv, kr, pc, dkr, dpc);
        } else {
            const double* w  = st + K.off_w[r];
            const double* g  = st + K.off_g[r];
            const double  Sg = in.S[n + c];
            const double  Sw = in.S[2 * n + c];
            double        v[4], s[4];
            eval_all(w, K.nrow_w[r], Sw, v, s);
            const double krw = v[1], dkrw = s[1], krow = v[2], dkrow = s[2];
            const double pcwo = -v[3], dpcw = -s[3];
            eval_all(g, K.nrow_g[r], Sg, v, s);
            const double krg = v[1], dkrg = s[1], krog = v[2], dkrog = s[2];
            const double pcgo = v[3], dpcg = s[3];
            // CalKro_Stone2 / CalKro_Stone2Der (src/FlowUnit.cpp:151-164, 301-328);
            // kroMax is SWOF's krow at its first row
            const double kmax = w[2 * K.nrow_w[r]];
            const double a1   = __dadd_rn(__ddiv_rn(krow, kmax), krw);
            const double a2   = __dadd_rn(__ddiv_rn(krog, kmax), krg);
            double       kro  = __dmul_rn(kmax, __dsub_rn(__dmul_rn(a1, a2), __dadd_rn(krw, krg)));
            double dkro_w = __dmul_rn(kmax, __dsub_rn(__dmul_rn(__dadd_rn(__ddiv_rn(dkrow, kmax), dkrw), a2), dkrw));
            double dkro_g = __dmul_rn(kmax, __dsub_rn(__dmul_rn(a1, __dadd_rn(__ddiv_rn(dkrog, kmax), dkrg)), dkrg));
            if (kro < 0) kro = dkro_w = dkro_g = 0;
            kr[0] = kro;
            kr[1] = krg;
            kr[2] = krw;
            pc[0] = 0;
            pc[1] = pcgo;
            pc[2] = pcwo;
#pragma unroll
            for (int j = 0; j < 9; j++) dkr[j] = dpc[j] = 0;
            dkr[1] = dkro_g;
            dkr[2] = dkro_w;
            dkr[4] = dkrg;
            dkr[8] = dkrw;
            dpc[4] = dpcg;
            dpc[8] = dpcw;
        }
        const double P = in.P[c];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            out.kr[j * n + c] = kr[j];
            out.Pc[j * n + c] = pc[j];
            out.Pj[j * n + c] = __dadd_rn(P, pc[j]);
        }
        if (deriv) {
#pragma unroll
            for (int j = 0; j < 9; j++) {
                out.dKr_dS[j * n + c]  = dkr[j];
                out.dPcj_dS[j * n + c] = dpc[j];
            }
        }
    }
}

}  // namespace
}  // namespace ocpf

struct ocpf_krpc {
    int             device;
    ocpf::KrpcConst k;
    double*         tab;
    int             blocks;
};

namespace ocpf {
namespace {

// Appends a table given row-major as its keyword lists it, column-major;
// false when it has fewer than 2 rows or its first column decreases (the
// table search relies on a non-decreasing column).
bool push_table(std::vector<double>& host, const double* rows, int nrow, int ncol, int32_t& off, int32_t& nr)
{
    if (!rows || nrow < 2) return false;
    for (int i = 1; i < nrow; i++)
        if (!(rows[ncol * i] >= rows[ncol * (i - 1)])) return false;
    off = (int32_t)host.size();
    nr  = nrow;
    for (int c = 0; c < ncol; c++)
        for (int i = 0; i < nrow; i++) host.push_back(rows[ncol * i + c]);
    return true;
}

int make_handle(KrpcConst& k, const std::vector<double>& host, int device, ocpf_krpc** out)
{
    if ((int64_t)host.size() > KRPC_MAX_DBL) return OCPF_EUNSUPPORTED;
    k.total  = (int32_t)host.size();
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return OCPF_ECUDA;
    int rc  = OCPF_OK;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    ocpf_krpc* h = new (std::nothrow) ocpf_krpc;
    if (!h) rc = OCPF_ENOMEM;
    if (rc == OCPF_OK) {
        h->device = device;
        h->k      = k;
        h->tab    = nullptr;
        h->blocks = (sms > 0 ? sms : 148) * 8;
        if (cudaMalloc(&h->tab, host.size() * sizeof(double)) != cudaSuccess)
            rc = OCPF_ENOMEM;
        else if (cudaMemcpy(h->tab, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice) !=
                 cudaSuccess)
            rc = OCPF_ECUDA;
    }
    if (rc != OCPF_OK && h) {
        if (h->tab) cudaFree(h->tab);
        delete h;
        h = nullptr;
    }
    if (prev != device) cudaSetDevice(prev);
    *out = h;
    return rc;
}

}  // namespace
}  // namespace ocpf

extern "C" int ocpf_krpc_create(const ocpf_satfunc* regions, int nregion, int device, ocpf_krpc** out)
{
    using namespace ocpf;
    if (!out) return OCPF_EINVAL;
    *out = nullptr;
    if (!regions || nregion < 1 || nregion > KRPC_MAX_REG) return OCPF_EINVAL;
    KrpcConst k;
    std::memset(&k, 0, sizeof(k));
    k.nreg   = nregion;
    k.family = KRPC_SWOF;
    std::vector<double> host;
    for (int r = 0; r < nregion; r++) {
        const ocpf_satfunc& f = regions[r];
        if (!push_table(host, f.swof, f.nrow_swof, 4, k.off_w[r], k.nrow_w[r]) ||
            !push_table(host, f.sgof, f.nrow_sgof, 4, k.off_g[r], k.nrow_g[r]))
            return OCPF_EINVAL;
    }
    return make_handle(k, host, device, out);
}

extern "C" int ocpf_krpc_create_sof3(const ocpf_satfunc3* regions, int nregion, int device, ocpf_krpc** out)
{
    using namespace ocpf;
    if (!out) return OCPF_EINVAL;
    *out = nullptr;
    if (!regions || nregion < 1 || nregion > KRPC_MAX_REG) return OCPF_EINVAL;
    KrpcConst k;
    std::memset(&k, 0, sizeof(k));
    k.nreg   = nregion;
    k.family = KRPC_SOF3;
    std::vector<double> host;
    for (int r = 0; r < nregion; r++) {
        const ocpf_satfunc3& f = regions[r];
        if (!push_table(host, f.swfn, f.nrow_swfn, 3, k.off_w[r], k.nrow_w[r]) ||
            !push_table(host, f.sgfn, f.nrow_sgfn, 3, k.off_g[r], k.nrow_g[r]) ||
            !push_table(host, f.sof3, f.nrow_sof3, 3, k.off_o[r], k.nrow_o[r]))
            return OCPF_EINVAL;
    }
    return make_handle(k, host, device, out);
}

extern "C" int ocpf_krpc_destroy(ocpf_krpc* h)
{
    if (!h) return OCPF_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    cudaFree(h->tab);
    if (prev != h->device) cudaSetDevice(prev);
    delete h;
    return OCPF_OK;
}

extern "C" int ocpf_cal_krpc(ocpf_krpc* h, int64_t ncell, const ocpf_krpc_in* in, const ocpf_krpc_out* out,
                         void* stream)
{
    using namespace ocpf;
    if (!h || ncell < 0 || !in || !out) return OCPF_EINVAL;
    if (ncell == 0) return OCPF_OK;
    if (!in->P || !in->S || !out->kr || !out->Pc || !out->Pj) return OCPF_EINVAL;
    if ((out->dKr_dS == nullptr) != (out->dPcj_dS == nullptr)) return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != h->device) cudaSetDevice(h->device);
    const int64_t need   = (ncell + KRPC_THREADS - 1) / KRPC_THREADS;
    const int     blocks = (int)(need < h->blocks ? need : h->blocks);
    k_krpc<<<blocks, KRPC_THREADS, h->k.total * sizeof(double), (cudaStream_t)stream>>>(h->k, h->tab, ncell, *in,
                                                                                         *out);
    const cudaError_t e = cudaGetLastError();
    if (prev != h->device) cudaSetDevice(prev);
    return e == cudaSuccess ? OCPF_OK : OCPF_ECUDA;
}
