// flash_learned.cuh -- the learned initialiser inside the fast form
// (OCPF_FORM_FAST): fresh cells (no last phase count) are run through the
// MLP on the tcgen05 tensor cores (learned_tc.cuh), 128 cells per CTA, one
// cell per thread. A cell whose
// predicted probability of ending two-phase reaches the confidence skips the
// stability test and goes straight to a split (round LEARN_ROUND); the
// rest, and every cell whose learned split fails its checks
// (learned_after_nr), take the strict stability test as in the other forms.
// The split starts from Wilson's K, not from the network's ln K: a different
// start can lead the substitution to a different solution where the
// mixture has more than one, and it shortens a linearly converging
// substitution by only a step or two. No counterpart in the reference.
#pragma once

#include "flash_phased.cuh"
#include "learned_tc.cuh"

namespace ocpf {

using LearnSmem = MlpTcSmem;
constexpr int LEARN_TILE = MLP_TC_ROWS;  // fresh cells per CTA tile

// One CTA of 128 threads takes the fresh-cell list in tiles of 128 cells,
// thread t the tile's cell t. Features: ln(P / psia), T / degF,
// z_1..z_NC, each normalised by the initialiser's mean and scale. A cell
// whose network output is not finite (the tensor-core pipeline did not
// answer) takes the stability test like a low-confidence one.
template <int NC>
__device__ void learn_body(const FluidConst& F, const PhasedArgs& a, LearnSmem& sm)
{
    using F_ = SF<NC>;
    static_assert(NC + 2 <= MLP_IO && NC + 1 <= MLP_IO, "network width");
    const StateBuf& S = a.S;
    const uint32_t  n = a.L.len(L_FRESH);
    MlpTc           net(sm);
    net.begin(a.mlp);
    for (uint32_t base = vblock(a) * (uint32_t)LEARN_TILE; base < n; base += vgrid(a) * (uint32_t)LEARN_TILE) {
        const uint32_t k = base + threadIdx.x;
        int64_t        c = -1;
        float          f[MLP_IO], o[MLP_IO];
#pragma unroll
        for (int j = 0; j < MLP_IO; j++) f[j] = 0.f;
        if (k < n) {
            c = a.L.item(L_FRESH, k);
            double z[NC];
            load_z<NC>(a, c, z);
            f[0] = (float)log(a.in.P[c]);
            f[1] = (float)a.in.T[c];
#pragma unroll
            for (int i = 0; i < NC; i++) f[2 + i] = (float)z[i];
#pragma unroll
            for (int j = 0; j < NC + 2; j++) f[j] = (f[j] - F.lin_mean[j]) / F.lin_scale[j];
        }
        net.forward(f, o);
        if (c >= 0) {
            const float pu = 1.f / (1.f + __expf(-o[0]));
            if (pu >= F.learn_conf) {
                // a two-phase start, as for a cell whose stability test
                // found it unstable with Yt < 1.1 (the tighter split
                // settings); the split starts from Wilson's K as the
                // reference's does (sp_prep), so it reaches the same
                // solution branch
                const uint32_t meta = (uint32_t)S.I(IF_META, c);
                S.D(F_::Yt, c)    = 1.01;
                S.I(IF_META, c)   = (int32_t)((meta & ~M_NP_MASK) | 2u | M_LEARNED);
                a.L.push(L_SP_LEARN, (int32_t)c);
            } else {
                a.L.push(L_STA_0, (int32_t)c);
            }
        }
    }
    net.end();
}

}  // namespace ocpf
